// (d1, d2) Smoothed-aggregation AMG preconditioner: host set-up of the hierarchy's
// structure, device numeric set-up on every value update, and the V-cycle apply.
//
// The reference preconditions DFGMRES with one BoomerAMG V-cycle
// (+LINEAR_SOLVERS/mex/hypre_boomeramg_mex.cpp:751-796, max_iter = 1, tol = 0) and re-runs the
// set-up after every value update (:1151-1213).  HYPRE is not part of this build; this is an
// AMG of its own design for the same role:
//
//   structure (host, once per pattern)   aggregation of the node-block graph, tentative
//       prolongator T from the near-null space (6 rigid-body modes in 3D, 3 in 2D) by a
//       per-aggregate QR, and fixed-pattern product plans for A T, A P and P' (A P)
//   numerics (device, every update)      block-Jacobi inverse, lambda_max(D^-1 A) by power
//       iteration (10 steps from a fixed vector at set-up and first update, then 3 more from
//       the previous vector at each later update), P = T - omega D^-1 A T (omega = 4 / (3 lambda_max)), R = P', A P,
//       A_c = P' (A P); coarsest level: dense Gauss-Jordan inverse
//   apply (device)                       V(1,1) cycle with degree-3 Chebyshev smoothing on
//       D^-1 A over [lambda_max / 10, 1.1 lambda_max], in FP64 or FP32 (mixed precision)
//
// Defaults (strength threshold 0.02 on every level, Chebyshev degree 3 on the interval ratio
// 10) were chosen on the SSR continuation of the 40 m slope: against threshold 0.05, degree 2
// and ratio 30 they cut the FGMRES iterations per continuation step from ~265 to ~36 and the
// step time about 4x.
//
// Every product is a gather over a precomputed list, so the numeric set-up uses no atomics
// and is deterministic.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <array>
#include <new>
#include <type_traits>
#include <vector>

#include "instr.cuh"
#include "linalg.cuh"
#include "mesh.h"
#include "sg_common.cuh"

namespace sg {

struct Pattern {  // CSR of blocks (rectangular)
    int64_t nrows = 0, ncols = 0, nblk = 0;
    std::vector<int32_t> rp, col;
    int32_t *d_rp = nullptr, *d_col = nullptr, *d_row = nullptr;  // d_row: block row of every block
};

struct Plan {  // for every output block: a list of (first, second) input block indices
    std::vector<int64_t> ptr;
    std::vector<int32_t> a, b;
    int64_t *d_ptr = nullptr;
    int32_t *d_a = nullptr, *d_b = nullptr;
};

struct Level {
    int b = 3, bc = 6;             // block size, coarse block size
    int64_t n = 0;                 // block rows
    const sg_bsr *Aext = nullptr;  // level 0: caller's pattern
    Pattern Aown;                  // coarse levels: own pattern
    const int32_t *d_Arp = nullptr, *d_Acol = nullptr, *d_Adiag = nullptr;
    int64_t Anblk = 0;
    const double *Avals = nullptr;  // level 0: caller's values (set at update)
    double *Aown_vals = nullptr;    // coarse levels
    float *A32 = nullptr;
    uint2 *A16 = nullptr;          // level 0 with fine_half: FP16 rows of A / a16_scale, 3 words per block
    float a16_scale = 1.0f;        // power of two putting the set-up matrix's largest entry near 4096
    int32_t *d_diag_own = nullptr;
    double *Dinv = nullptr;
    float *Dinv32 = nullptr;
    double *lmax = nullptr;        // device scalar
    uint8_t *d_dead = nullptr;     // per DOF: dead coarse DOF (identity row), coarse levels only
    // transfer to the next level
    std::vector<int32_t> agg;
    int32_t *d_agg = nullptr;
    double *T = nullptr;           // n * b * bc
    Pattern P, R, AP;
    int32_t *d_R_from_P = nullptr;
    Plan at_plan, ap_plan, ac_plan;  // at: (A block) per P block; ap: (A, P); ac: (P, AP)
    int64_t ap_pairs = 0, ac_pairs = 0;  // plan lengths (pairs of input blocks)
    // symmetric Galerkin product (option symmetric): ac_plan covers the coarse blocks (I, J)
    // with I <= J only, d_ac_out[t] being their indices in the coarse pattern; the blocks
    // below the diagonal are copied transposed from d_ac_lower_src into d_ac_lower
    int64_t n_ac_items = 0, n_ac_lower = 0;
    int32_t *d_ac_out = nullptr, *d_ac_lower = nullptr, *d_ac_lower_src = nullptr;
    double *Pv = nullptr, *Rv = nullptr, *APv = nullptr;
    float *P32 = nullptr, *R32 = nullptr;
    float *T32 = nullptr, *APv32 = nullptr;   // mixed form: FP32 numeric updates
    // vectors
    double *x = nullptr, *rhs = nullptr, *r = nullptr, *d = nullptr, *t = nullptr;
    double *pv = nullptr;          // power-iteration vector, kept between updates
    int power_warm = 0;            // numeric passes done on this level (warm start from the third)
    float *x32 = nullptr, *rhs32 = nullptr, *r32 = nullptr, *d32 = nullptr;
};

struct AmgOptions {
    int max_levels = 10;
    int coarse_size = 1200;   // stop coarsening at this many DOFs
    int cheb_degree = 3;
    double cheb_ratio = 10.0; // smoothing interval [lmax / ratio, 1.1 lmax]
    int power_its = 10;       // first set-up; later updates continue from the last vector:
    int power_its_warm = 3;   // lambda_max moves little between Newton iterations
    int mixed = 0;            // 1: FP32 V-cycle
    double omega_scale = 4.0 / 3.0;
    double theta = 0.02;      // strength threshold (0: whole block graph)
    int fine_half = 0;        // mixed form, 3x3 level 0: the cycle's level-0 SpMVs read an FP16 copy
    int symmetric = 0;        // 1: A is symmetric, so every Galerkin matrix P'AP is: only its blocks
                              // on and above the diagonal are formed, the others mirrored
};

}  // namespace sg

struct sg_amg {
    sg::AmgOptions opt;
    std::vector<sg::Level> L;
    int64_t nc_dense = 0;      // coarsest dense size (DOFs)
    double *Ainv = nullptr;    // dense inverse, nc_dense^2
    float *Ainv32 = nullptr;
    double *colk = nullptr, *rowk = nullptr;   // Gauss-Jordan column block (N x NB) and row block (NB x N)
    double *gj_pinv = nullptr;                 // inverse of the current pivot block (NB x NB)
    double *dots = nullptr;    // reduction scratch
    // optional node-wise correction after the cycle: z += C (r - A z), C n x 3 x 3 (3D only)
    double *corrC = nullptr;
    float *corrC32 = nullptr;
    int corr_on = 0;
    int device = 0;
    int updated = 0;
    // a clone (sg_amg_clone) shares every matrix, transfer operator and inverse of its parent
    // and owns only its cycle vectors
    const sg_amg *parent = nullptr;
};

namespace sg {

template <typename T>
static int dalloc(T **p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    SG_CUDA(sg::device_alloc((void **)p, n * sizeof(T)));
    return SG_OK;
}
template <typename T>
static int dup(T **p, const std::vector<T> &v) {
    int rc = dalloc(p, v.size());
    if (rc) return rc;
    if (!v.empty()) SG_CUDA(cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return SG_OK;
}

// ------------------------------------------------------------------ host structure set-up

// Three-phase aggregation of the block graph (rp, col), rows with active[i] == 0 excluded.
static int64_t aggregate(int64_t n, const std::vector<int32_t> &rp, const std::vector<int32_t> &col,
                         const std::vector<uint8_t> &active, std::vector<int32_t> &agg) {
    agg.assign(n, -1);
    int32_t na = 0;
    for (int64_t i = 0; i < n; ++i) {  // phase 1: roots whose neighbourhood is untouched
        if (!active[i] || agg[i] >= 0) continue;
        bool free_nb = true;
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            const int32_t j = col[p];
            if (active[j] && agg[j] >= 0) { free_nb = false; break; }
        }
        if (!free_nb) continue;
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            const int32_t j = col[p];
            if (active[j]) agg[j] = na;
        }
        agg[i] = na++;
    }
    std::vector<int32_t> add(n, -1);
    for (int64_t i = 0; i < n; ++i) {  // phase 2: join the neighbouring aggregate seen most
        if (!active[i] || agg[i] >= 0) continue;
        int32_t best = -1, bestc = 0;
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            const int32_t a = agg[col[p]];
            if (a < 0) continue;
            int32_t c = 0;
            for (int32_t q = rp[i]; q < rp[i + 1]; ++q) c += (agg[col[q]] == a);
            if (c > bestc) { bestc = c; best = a; }
        }
        add[i] = best;
    }
    for (int64_t i = 0; i < n; ++i)
        if (add[i] >= 0) agg[i] = add[i];
    for (int64_t i = 0; i < n; ++i) {  // phase 3: leftovers form their own aggregates
        if (!active[i] || agg[i] >= 0) continue;
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            const int32_t j = col[p];
            if (active[j] && agg[j] < 0) agg[j] = na;
        }
        agg[i] = na++;
    }
    return na;
}

// Per-aggregate thin QR (modified Gram-Schmidt, two passes) of the near-null space rows.
// B: n*b rows x k columns (row-major).  Outputs T (n*b x k), Bc (na*k x k) and dead flags.
static void tentative(int64_t n, int b, int k, int64_t na, const std::vector<int32_t> &agg,
                      const std::vector<double> &B, std::vector<double> &T, std::vector<double> &Bc,
                      std::vector<uint8_t> &dead) {
    std::vector<std::vector<int32_t>> members(na);
    for (int64_t i = 0; i < n; ++i)
        if (agg[i] >= 0) members[agg[i]].push_back((int32_t)i);
    T.assign((size_t)n * b * k, 0.0);
    Bc.assign((size_t)na * k * k, 0.0);
    dead.assign((size_t)na * k, 0);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t a = 0; a < na; ++a) {
        const auto &mem = members[a];
        const int m = (int)mem.size() * b;
        std::vector<double> Qm((size_t)m * k), Rm((size_t)k * k, 0.0);
        for (int r = 0; r < m; ++r) {
            const int64_t row = (int64_t)mem[r / b] * b + r % b;
            for (int c = 0; c < k; ++c) Qm[(size_t)r * k + c] = B[(size_t)row * k + c];
        }
        double scale = 0.0;
        for (double v : Qm) scale = std::max(scale, std::fabs(v));
        for (int c = 0; c < k; ++c) {
            double nrm0 = 0.0;
            for (int r = 0; r < m; ++r) nrm0 += Qm[(size_t)r * k + c] * Qm[(size_t)r * k + c];
            nrm0 = std::sqrt(nrm0);
            for (int pass = 0; pass < 2; ++pass) {
                for (int c2 = 0; c2 < c; ++c2) {
                    double h = 0.0;
                    for (int r = 0; r < m; ++r) h += Qm[(size_t)r * k + c2] * Qm[(size_t)r * k + c];
                    for (int r = 0; r < m; ++r) Qm[(size_t)r * k + c] -= h * Qm[(size_t)r * k + c2];
                    Rm[(size_t)c2 * k + c] += h;
                }
            }
            double nrm = 0.0;
            for (int r = 0; r < m; ++r) nrm += Qm[(size_t)r * k + c] * Qm[(size_t)r * k + c];
            nrm = std::sqrt(nrm);
            if (nrm <= 1e-10 * std::max(nrm0, scale * 1e-3) || nrm == 0.0) {
                for (int r = 0; r < m; ++r) Qm[(size_t)r * k + c] = 0.0;
                for (int c2 = 0; c2 < k; ++c2) Rm[(size_t)c * k + c2] = 0.0;
                dead[(size_t)a * k + c] = 1;
                continue;
            }
            Rm[(size_t)c * k + c] = nrm;
            for (int r = 0; r < m; ++r) Qm[(size_t)r * k + c] /= nrm;
        }
        for (int r = 0; r < m; ++r) {
            const int64_t row = (int64_t)mem[r / b] * b + r % b;
            for (int c = 0; c < k; ++c) T[(size_t)row * k + c] = Qm[(size_t)r * k + c];
        }
        for (size_t t = 0; t < Rm.size(); ++t) Bc[(size_t)a * k * k + t] = Rm[t];
    }
}

// Row-wise symbolic product helper: for each row, collect (col, a, b) triples, sort by col,
// emit the pattern row and the plan (list of (a, b) per output block).
template <typename F>
static void build_product(int64_t nrows, Pattern &out, Plan &plan, F collect) {
    std::vector<std::vector<int32_t>> cols(nrows);
    std::vector<std::vector<int64_t>> cnt(nrows);
    std::vector<std::vector<int32_t>> la(nrows), lb(nrows);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < nrows; ++i) {
        std::vector<std::array<int32_t, 3>> tr;
        collect(i, tr);
        std::sort(tr.begin(), tr.end());
        auto &c = cols[i];
        auto &n = cnt[i];
        auto &A = la[i];
        auto &B = lb[i];
        for (size_t t = 0; t < tr.size(); ++t) {
            if (c.empty() || c.back() != tr[t][0]) {
                c.push_back(tr[t][0]);
                n.push_back(0);
            }
            n.back()++;
            A.push_back(tr[t][1]);
            B.push_back(tr[t][2]);
        }
    }
    out.nrows = nrows;
    out.rp.assign(nrows + 1, 0);
    for (int64_t i = 0; i < nrows; ++i) out.rp[i + 1] = out.rp[i] + (int32_t)cols[i].size();
    out.nblk = out.rp[nrows];
    out.col.resize(out.nblk);
    plan.ptr.assign(out.nblk + 1, 0);
    for (int64_t i = 0; i < nrows; ++i)
        for (size_t t = 0; t < cols[i].size(); ++t) plan.ptr[out.rp[i] + t + 1] = cnt[i][t];
    for (int64_t p = 0; p < out.nblk; ++p) plan.ptr[p + 1] += plan.ptr[p];
    plan.a.resize(plan.ptr[out.nblk]);
    plan.b.resize(plan.ptr[out.nblk]);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < nrows; ++i) {
        std::copy(cols[i].begin(), cols[i].end(), out.col.begin() + out.rp[i]);
        const int64_t base = plan.ptr[out.rp[i]];
        std::copy(la[i].begin(), la[i].end(), plan.a.begin() + base);
        std::copy(lb[i].begin(), lb[i].end(), plan.b.begin() + base);
        std::vector<int32_t>().swap(cols[i]);
        std::vector<int32_t>().swap(la[i]);
        std::vector<int32_t>().swap(lb[i]);
    }
}

static int upload_pattern(Pattern &p) {
    std::vector<int32_t> row(p.col.size());
    for (int64_t i = 0; i < (int64_t)p.rp.size() - 1; ++i)
        for (int32_t q = p.rp[i]; q < p.rp[i + 1]; ++q) row[q] = (int32_t)i;
    int rc = dup(&p.d_rp, p.rp);
    if (!rc) rc = dup(&p.d_col, p.col);
    if (!rc) rc = dup(&p.d_row, row);
    return rc;
}
static int upload_plan(Plan &p) {
    int rc = dup(&p.d_ptr, p.ptr);
    if (!rc) rc = dup(&p.d_a, p.a);
    if (!rc) rc = dup(&p.d_b, p.b);
    return rc;
}

// ------------------------------------------------------------------ device numerics

// In-register Gauss-Jordan inverse of a small SPD block (no pivoting needed for SPD).
template <int B>
__device__ __forceinline__ void inv_block(const double *a, double *out) {
    double m[B][2 * B];
#pragma unroll
    for (int i = 0; i < B; ++i)
#pragma unroll
        for (int j = 0; j < B; ++j) {
            m[i][j] = a[i * B + j];
            m[i][B + j] = (i == j) ? 1.0 : 0.0;
        }
#pragma unroll
    for (int k = 0; k < B; ++k) {
        const double piv = m[k][k];
        const double ip = (piv != 0.0) ? 1.0 / piv : 0.0;
#pragma unroll
        for (int j = 0; j < 2 * B; ++j) m[k][j] *= ip;
#pragma unroll
        for (int i = 0; i < B; ++i) {
            if (i == k) continue;
            const double f = m[i][k];
#pragma unroll
            for (int j = 0; j < 2 * B; ++j) m[i][j] -= f * m[k][j];
        }
    }
#pragma unroll
    for (int i = 0; i < B; ++i)
#pragma unroll
        for (int j = 0; j < B; ++j) out[i * B + j] = m[i][B + j];
}

template <int B, typename V = double>
__global__ void k_block_diag_inv(int64_t n, const int32_t *__restrict__ diag, const V *__restrict__ A,
                                 double *__restrict__ Dinv, float *__restrict__ Dinv32) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double a[B * B], o[B * B];
        const int64_t p = diag[i];
#pragma unroll
        for (int t = 0; t < B * B; ++t) a[t] = (p >= 0) ? (double)A[p * B * B + t] : ((t % (B + 1)) == 0 ? 1.0 : 0.0);
        inv_block<B>(a, o);
#pragma unroll
        for (int t = 0; t < B * B; ++t) {
            Dinv[i * B * B + t] = o[t];
            if (Dinv32) Dinv32[i * B * B + t] = (float)o[t];
        }
    }
}

// y = Dinv x (blockwise), optionally scaled by s (device scalar, inverted when inv != 0)
template <int B, typename T>
__global__ void k_dinv_apply(int64_t n, const T *__restrict__ Dinv, const T *__restrict__ x, T *__restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        T xv[B];
#pragma unroll
        for (int b = 0; b < B; ++b) xv[b] = x[i * B + b];
#pragma unroll
        for (int a = 0; a < B; ++a) {
            T s = 0;
#pragma unroll
            for (int b = 0; b < B; ++b) s += Dinv[(i * B + a) * B + b] * xv[b];
            y[i * B + a] = s;
        }
    }
}

// Chebyshev step on D^-1 A with bounds [lmax/ratio, 1.1 lmax]:
//   first (k == 0):  d = D^-1 r / theta;               x += d
//   next  (k >= 1):  d = c1 d + c2 D^-1 r;             x += d
// rho_k follows rho_0 = 1/sigma, rho_{k} = 1/(2 sigma - rho_{k-1}).
template <int B, typename T>
__global__ void k_cheb(int64_t n, int k, double ratio, const double *__restrict__ lmax, const T *__restrict__ Dinv,
                       const T *__restrict__ r, T *__restrict__ d, T *__restrict__ x, int x_is_zero) {
    const double hi = 1.1 * lmax[0], lo = lmax[0] / ratio;
    const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
    double rho = 1.0 / sigma, c1 = 0.0, c2 = 1.0 / theta;
    for (int s = 1; s <= k; ++s) {
        const double rn = 1.0 / (2.0 * sigma - rho);
        c1 = rn * rho;
        c2 = 2.0 * rn / delta;
        rho = rn;
    }
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        T rv[B];
#pragma unroll
        for (int b = 0; b < B; ++b) rv[b] = r[i * B + b];
#pragma unroll
        for (int a = 0; a < B; ++a) {
            T s = 0;
#pragma unroll
            for (int b = 0; b < B; ++b) s += Dinv[(i * B + a) * B + b] * rv[b];
            const T dn = (k == 0) ? (T)c2 * s : (T)c1 * d[i * B + a] + (T)c2 * s;
            d[i * B + a] = dn;
            x[i * B + a] = (x_is_zero && k == 0) ? dn : x[i * B + a] + dn;
        }
    }
}

// P block (i,J) = [agg(i) == J] T_i - omega Dinv_i sum_{p in list} A_p T_{col(p)},  omega = s / lmax
// One thread per P block.
template <int B, int BC, typename V = double>
__global__ void k_smooth_prolongator(int64_t nblk, const int32_t *__restrict__ Prow, const int32_t *__restrict__ Pcol,
                                     const int64_t *__restrict__ lptr, const int32_t *__restrict__ la,
                                     const int32_t *__restrict__ Acol, const V *__restrict__ A,
                                     const V *__restrict__ T, const int32_t *__restrict__ agg,
                                     const double *__restrict__ Dinv, const double *__restrict__ lmax, double oscale,
                                     V *__restrict__ P, int64_t chunk) {
    const double omega = oscale / lmax[0];
    const int64_t q0 = (int64_t)blockIdx.x * chunk, q1 = q0 + chunk < nblk ? q0 + chunk : nblk;
    for (int64_t q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
        const int64_t i = Prow[q];
        {
            double acc[B * BC];
#pragma unroll
            for (int t = 0; t < B * BC; ++t) acc[t] = 0.0;
            for (int64_t l = lptr[q]; l < lptr[q + 1]; ++l) {
                const int32_t p = la[l];
                const V *a = A + (int64_t)p * B * B;
                const V *tk = T + (int64_t)Acol[p] * B * BC;
#pragma unroll
                for (int r = 0; r < B; ++r)
#pragma unroll
                    for (int m = 0; m < B; ++m) {
                        const double av = (double)a[r * B + m];
#pragma unroll
                        for (int c = 0; c < BC; ++c) acc[r * BC + c] += av * (double)tk[m * BC + c];
                    }
            }
            const double *di = Dinv + i * B * B;
            const bool own = agg[i] == Pcol[q];
            const V *ti = T + i * B * BC;
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int c = 0; c < BC; ++c) {
                    double s = 0.0;
#pragma unroll
                    for (int m = 0; m < B; ++m) s += di[r * B + m] * acc[m * BC + c];
                    P[(int64_t)q * B * BC + r * BC + c] = (V)((own ? (double)ti[r * BC + c] : 0.0) - omega * s);
                }
        }
    }
}

// R block k = transpose of P block from[k]
template <int B, int BC, typename V = double>
__global__ void k_transpose_blocks(int64_t nblk, const int32_t *__restrict__ from, const V *__restrict__ P,
                                   V *__restrict__ R) {
    const int64_t total = nblk * B * BC;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = t / (B * BC);
        const int e = (int)(t - k * B * BC), c = e / B, r = e - c * B;  // R(c, r) = P(r, c)
        R[t] = P[(int64_t)from[k] * B * BC + r * BC + c];
    }
}

// Block of N doubles into registers: pairs of 16-byte loads when N is even (blocks of such
// arrays then start on 16-byte boundaries), single loads otherwise.
template <int N>
__device__ __forceinline__ void load_block(const double *__restrict__ src, double *dst) {
    if constexpr (N % 2 == 0) {
        const double2 *s2 = reinterpret_cast<const double2 *>(src);
#pragma unroll
        for (int t = 0; t < N / 2; ++t) {
            const double2 w = __ldg(s2 + t);
            dst[2 * t] = w.x;
            dst[2 * t + 1] = w.y;
        }
    } else {
#pragma unroll
        for (int t = 0; t < N; ++t) dst[t] = __ldg(src + t);
    }
}
// FP32 blocks (the mixed-precision set-up): pairs of 8-byte loads when N is even
template <int N>
__device__ __forceinline__ void load_block(const float *__restrict__ src, double *dst) {
    if constexpr (N % 2 == 0) {
        const float2 *s2 = reinterpret_cast<const float2 *>(src);
#pragma unroll
        for (int t = 0; t < N / 2; ++t) {
            const float2 w = __ldg(s2 + t);
            dst[2 * t] = w.x;
            dst[2 * t + 1] = w.y;
        }
    } else {
#pragma unroll
        for (int t = 0; t < N; ++t) dst[t] = __ldg(src + t);
    }
}

// Block of N values in their storage type into registers (16-byte loads when the block size
// allows it; blocks of such arrays then start on 16-byte boundaries).
template <int N, typename V>
__device__ __forceinline__ void load_raw(const V *__restrict__ src, V *dst) {
    constexpr int W = 16 / (int)sizeof(V);
    if constexpr (N % W == 0) {
        using Vec = typename std::conditional<sizeof(V) == 8, double2, float4>::type;
        const Vec *s = reinterpret_cast<const Vec *>(src);
#pragma unroll
        for (int t = 0; t < N / W; ++t) *reinterpret_cast<Vec *>(dst + t * W) = __ldg(s + t);
    } else if constexpr (sizeof(V) == 4 && N % 2 == 0) {
        const float2 *s = reinterpret_cast<const float2 *>(src);
#pragma unroll
        for (int t = 0; t < N / 2; ++t) *reinterpret_cast<float2 *>(dst + 2 * t) = __ldg(s + t);
    } else {
#pragma unroll
        for (int t = 0; t < N; ++t) dst[t] = __ldg(src + t);
    }
}

// Accumulator type of the Galerkin gathers: FP64 for the FP64 set-up, FP32 for the FP32 one
// (the mixed form's coarse operators are stored in FP32 anyway).
template <typename V> struct GAcc { using type = double; };
template <> struct GAcc<float> { using type = float; };

// AP block = sum over plan pairs A_a (B x B) * P_b (B x BC), one thread per AP block.  For the
// small block shapes two pairs are in flight per iteration (their index and block loads
// issued before either product), which doubles the loads a thread keeps outstanding; the
// products are added in pair order, as with one pair per iteration.
template <int B, int BC, typename V = double>
__global__ void k_gather_AP(int64_t nblk, const int64_t *__restrict__ lptr, const int32_t *__restrict__ la,
                            const int32_t *__restrict__ lb, const V *__restrict__ A, const V *__restrict__ P,
                            V *__restrict__ AP, int64_t chunk) {
    using T = typename GAcc<V>::type;
    const int64_t q0 = (int64_t)blockIdx.x * chunk, q1 = q0 + chunk < nblk ? q0 + chunk : nblk;
    for (int64_t q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
        T acc[B * BC];
#pragma unroll
        for (int t = 0; t < B * BC; ++t) acc[t] = 0;
        const int64_t l1 = lptr[q + 1];
        int64_t l = lptr[q];
        auto product = [&](const V *a, const V *pv) {
#pragma unroll
            for (int r = 0; r < B; ++r)
#pragma unroll
                for (int m = 0; m < B; ++m) {
                    const T av = (T)a[r * B + m];
#pragma unroll
                    for (int c = 0; c < BC; ++c) acc[r * BC + c] += av * (T)pv[m * BC + c];
                }
        };
        if constexpr (B * B + B * BC <= 27) {   // two pairs in flight (fine level and 2D shapes)
            for (; l + 1 < l1; l += 2) {
                const int64_t ia0 = la[l], ib0 = lb[l], ia1 = la[l + 1], ib1 = lb[l + 1];
                V a0[B * B], p0[B * BC], a1[B * B], p1[B * BC];
                load_raw<B * B>(A + ia0 * B * B, a0);
                load_raw<B * BC>(P + ib0 * B * BC, p0);
                load_raw<B * B>(A + ia1 * B * B, a1);
                load_raw<B * BC>(P + ib1 * B * BC, p1);
                product(a0, p0);
                product(a1, p1);
            }
        }
        for (; l < l1; ++l) {
            V a0[B * B], p0[B * BC];
            load_raw<B * B>(A + (int64_t)la[l] * B * B, a0);
            load_raw<B * BC>(P + (int64_t)lb[l] * B * BC, p0);
            product(a0, p0);
        }
#pragma unroll
        for (int t = 0; t < B * BC; ++t) AP[q * B * BC + t] = (V)acc[t];
    }
}

// Ac block (I,J) = sum over plan pairs P_a' (BC x B) * AP_b (B x BC); dead DOFs get identity.
// One thread per coarse block.
// With qmap (symmetric Galerkin product) item t of the plan is coarse block qmap[t].
template <int B, int BC, typename V = double>
__global__ void k_gather_Ac(int64_t nitems, const int32_t *__restrict__ qmap, const int32_t *__restrict__ row,
                            const int32_t *__restrict__ col, const int64_t *__restrict__ lptr,
                            const int32_t *__restrict__ la, const int32_t *__restrict__ lb,
                            const V *__restrict__ P, const V *__restrict__ AP, const uint8_t *__restrict__ dead,
                            V *__restrict__ Ac, int64_t chunk) {
    const int64_t i0 = (int64_t)blockIdx.x * chunk, i1 = i0 + chunk < nitems ? i0 + chunk : nitems;
    for (int64_t it = i0 + threadIdx.x; it < i1; it += blockDim.x) {
        const int64_t q = qmap ? (int64_t)qmap[it] : it;
        const int64_t I = row[q];
        {
            const int64_t J = col[q];
            double acc[BC * BC];
#pragma unroll
            for (int t = 0; t < BC * BC; ++t) acc[t] = 0.0;
            for (int64_t l = lptr[it]; l < lptr[it + 1]; ++l) {
                double p[B * BC], ap[B * BC];
                load_block<B * BC>(P + (int64_t)la[l] * B * BC, p);
                load_block<B * BC>(AP + (int64_t)lb[l] * B * BC, ap);
#pragma unroll
                for (int m = 0; m < B; ++m)
#pragma unroll
                    for (int r = 0; r < BC; ++r) {
                        const double pv = p[m * BC + r];
#pragma unroll
                        for (int c = 0; c < BC; ++c) acc[r * BC + c] += pv * ap[m * BC + c];
                    }
            }
#pragma unroll
            for (int r = 0; r < BC; ++r)
#pragma unroll
                for (int c = 0; c < BC; ++c) {
                    double v = acc[r * BC + c];
                    if (dead[I * BC + r] || dead[J * BC + c]) v = (I == J && r == c) ? 1.0 : 0.0;
                    Ac[(int64_t)q * BC * BC + r * BC + c] = (V)v;
                }
        }
    }
}

// Lane-group variants of the two gathers for output blocks that each sum many pairs (the
// coarse levels, and P'(AP) on the fine level): G lanes (8, 16 or 32) share one output block,
// split its pairs and combine their partial sums by a fixed shuffle tree (deterministic).
// Fewer lanes per block mean more pairs per lane between the log2(G) shuffle steps, whose
// cost per output entry is fixed.
template <int B, int BC, typename V = double, int G = 32>
__global__ void k_gather_AP_warp(int64_t nblk, const int64_t *__restrict__ lptr, const int32_t *__restrict__ la,
                                 const int32_t *__restrict__ lb, const V *__restrict__ A,
                                 const V *__restrict__ P, V *__restrict__ AP, int64_t chunk) {
    const int lane = threadIdx.x & 31, gl = lane % G;
    // a CTA owns `chunk` consecutive output blocks (a multiple of its blockDim / G groups), so
    // every lane of a warp runs the same number of outer iterations (the shuffles need them)
    const int64_t c0 = (int64_t)blockIdx.x * chunk, c1 = c0 + chunk < nblk ? c0 + chunk : nblk;
    for (int64_t q = c0 + threadIdx.x / G; q < c0 + chunk; q += blockDim.x / G) {
        const bool live = q < c1;
        typename GAcc<V>::type acc[B * BC];
#pragma unroll
        for (int t = 0; t < B * BC; ++t) acc[t] = 0;
        if (live) {
            for (int64_t l = lptr[q] + gl; l < lptr[q + 1]; l += G) {
                V a[B * B], p[B * BC];
                load_raw<B * B>(A + (int64_t)la[l] * B * B, a);
                load_raw<B * BC>(P + (int64_t)lb[l] * B * BC, p);
#pragma unroll
                for (int r = 0; r < B; ++r)
#pragma unroll
                    for (int m = 0; m < B; ++m)
#pragma unroll
                        for (int c = 0; c < BC; ++c) acc[r * BC + c] += a[r * B + m] * p[m * BC + c];
            }
        }
#pragma unroll
        for (int t = 0; t < B * BC; ++t)
#pragma unroll
            for (int off = G / 2; off > 0; off >>= 1) acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], off);
        if (live && gl == 0)
#pragma unroll
            for (int t = 0; t < B * BC; ++t) AP[q * B * BC + t] = (V)acc[t];
    }
}

template <int B, int BC, typename V = double, int G = 32>
__global__ void k_gather_Ac_warp(int64_t nitems, const int32_t *__restrict__ qmap, const int32_t *__restrict__ row,
                                 const int32_t *__restrict__ col, const int64_t *__restrict__ lptr,
                                 const int32_t *__restrict__ la, const int32_t *__restrict__ lb,
                                 const V *__restrict__ P, const V *__restrict__ AP,
                                 const uint8_t *__restrict__ dead, V *__restrict__ Ac, int64_t chunk) {
    const int lane = threadIdx.x & 31, gl = lane % G;
    const int64_t c0 = (int64_t)blockIdx.x * chunk, c1 = c0 + chunk < nitems ? c0 + chunk : nitems;
    for (int64_t it = c0 + threadIdx.x / G; it < c0 + chunk; it += blockDim.x / G) {
        const bool live = it < c1;
        typename GAcc<V>::type acc[BC * BC];
#pragma unroll
        for (int t = 0; t < BC * BC; ++t) acc[t] = 0;
        if (live) {
            for (int64_t l = lptr[it] + gl; l < lptr[it + 1]; l += G) {
                V p[B * BC], ap[B * BC];
                load_raw<B * BC>(P + (int64_t)la[l] * B * BC, p);
                load_raw<B * BC>(AP + (int64_t)lb[l] * B * BC, ap);
#pragma unroll
                for (int m = 0; m < B; ++m)
#pragma unroll
                    for (int r = 0; r < BC; ++r)
#pragma unroll
                        for (int c = 0; c < BC; ++c) acc[r * BC + c] += p[m * BC + r] * ap[m * BC + c];
            }
        }
#pragma unroll
        for (int t = 0; t < BC * BC; ++t)
#pragma unroll
            for (int off = G / 2; off > 0; off >>= 1) acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], off);
        if (live && gl == 0) {
            const int64_t q = qmap ? (int64_t)qmap[it] : it;
            const int64_t I = row[q], J = col[q];
#pragma unroll
            for (int r = 0; r < BC; ++r)
#pragma unroll
                for (int c = 0; c < BC; ++c) {
                    double v = acc[r * BC + c];
                    if (dead[I * BC + r] || dead[J * BC + c]) v = (I == J && r == c) ? 1.0 : 0.0;
                    Ac[(int64_t)q * BC * BC + r * BC + c] = (V)v;
                }
        }
    }
}

// lanes per output block for the lane-group gathers: about 8 or more pairs per lane
inline int gather_lanes(int64_t nblk, int64_t pairs) {
    const double avg = nblk > 0 ? (double)pairs / (double)nblk : 0.0;
    return avg >= 256.0 ? 32 : (avg >= 128.0 ? 16 : 8);
}

template <int B, int BC, typename V>
static void gather_AP_groups(int64_t nblk, int64_t pairs, const int64_t *ptr, const int32_t *la, const int32_t *lb,
                             const V *A, const V *P, V *AP, cudaStream_t st) {
    const int G = gather_lanes(nblk, pairs);
    const int64_t ch = chunk_len(nblk, 128 / G, 8 * 128 / G);
    const unsigned grid = grid_chunks(nblk, ch);
    switch (G) {
        case 32: k_gather_AP_warp<B, BC, V, 32><<<grid, 128, 0, st>>>(nblk, ptr, la, lb, A, P, AP, ch); break;
        case 16: k_gather_AP_warp<B, BC, V, 16><<<grid, 128, 0, st>>>(nblk, ptr, la, lb, A, P, AP, ch); break;
        default: k_gather_AP_warp<B, BC, V, 8><<<grid, 128, 0, st>>>(nblk, ptr, la, lb, A, P, AP, ch); break;
    }
}

template <int B, int BC, typename V>
static void gather_Ac_groups(int64_t nitems, int64_t pairs, const int32_t *qmap, const int32_t *row,
                             const int32_t *col, const int64_t *ptr, const int32_t *la, const int32_t *lb, const V *P,
                             const V *AP, const uint8_t *dead, V *Ac, cudaStream_t st) {
    const int G = gather_lanes(nitems, pairs);
    const int64_t ch = chunk_len(nitems, 128 / G, 8 * 128 / G);
    const unsigned grid = grid_chunks(nitems, ch);
    switch (G) {
        case 32: k_gather_Ac_warp<B, BC, V, 32><<<grid, 128, 0, st>>>(nitems, qmap, row, col, ptr, la, lb, P, AP, dead, Ac, ch); break;
        case 16: k_gather_Ac_warp<B, BC, V, 16><<<grid, 128, 0, st>>>(nitems, qmap, row, col, ptr, la, lb, P, AP, dead, Ac, ch); break;
        default: k_gather_Ac_warp<B, BC, V, 8><<<grid, 128, 0, st>>>(nitems, qmap, row, col, ptr, la, lb, P, AP, dead, Ac, ch); break;
    }
}

// Blocks below the diagonal of a symmetric Galerkin matrix: A(dst) = A(src)'.
template <int BC, typename V>
__global__ void k_mirror_blocks(int64_t n, const int32_t *__restrict__ dst, const int32_t *__restrict__ src,
                                V *__restrict__ A) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const V *a = A + (int64_t)src[t] * BC * BC;
        V *o = A + (int64_t)dst[t] * BC * BC;
#pragma unroll
        for (int r = 0; r < BC; ++r)
#pragma unroll
            for (int c = 0; c < BC; ++c) o[r * BC + c] = a[c * BC + r];
    }
}

// P'(A P) into the next level's values: every block, or (symmetric) the blocks on and
// above the diagonal followed by the mirrored ones
template <int B, int BC, typename V>
static void galerkin_Ac(const Level &L, const Level &C, const V *P, const V *AP, V *Ac, cudaStream_t st) {
    const bool sym = L.d_ac_out != nullptr;
    const int64_t items = sym ? L.n_ac_items : C.Anblk;
    const int32_t *qmap = sym ? L.d_ac_out : nullptr;
    // one thread per output block, or a group of lanes per block where blocks are few or
    // each sums many pairs (on the SSR hierarchy: fine-level P'(A P), ~63 pairs per block,
    // 1.3x faster per lane group; the small coarse levels 10-20x faster)
    if (!(items < 32768 || L.ac_pairs >= 24 * items)) {
        const int64_t ch = chunk_len(items, 128, 8 * 128);
        k_gather_Ac<B, BC, V><<<grid_chunks(items, ch), 128, 0, st>>>(items, qmap, C.Aown.d_row, C.d_Acol,
                                                                      L.ac_plan.d_ptr, L.ac_plan.d_a, L.ac_plan.d_b,
                                                                      P, AP, C.d_dead, Ac, ch);
    } else
        gather_Ac_groups<B, BC, V>(items, L.ac_pairs, qmap, C.Aown.d_row, C.d_Acol, L.ac_plan.d_ptr, L.ac_plan.d_a,
                                   L.ac_plan.d_b, P, AP, C.d_dead, Ac, st);
    if (sym && L.n_ac_lower > 0)
        k_mirror_blocks<BC, V><<<grid_for(L.n_ac_lower, 256), 256, 0, st>>>(L.n_ac_lower, L.d_ac_lower,
                                                                           L.d_ac_lower_src, Ac);
}

__global__ void k_to_float(int64_t n, const double *__restrict__ a, float *__restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}
__global__ void k_to_double(int64_t n, const float *__restrict__ a, double *__restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}

// deterministic pseudo-random start vector for the power iteration
__global__ void k_init_vec(int64_t n, double *__restrict__ v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t h = (uint64_t)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
        h ^= h >> 31;
        h *= 0xBF58476D1CE4E5B9ull;
        h ^= h >> 29;
        v[i] = 0.5 + (double)(h >> 11) * (1.0 / 9007199254740992.0);
    }
}

// lmax = sqrt(dots[0]) ; v = w / lmax
__global__ void k_power_norm(int64_t n, const double *__restrict__ w, const double *__restrict__ dots,
                             double *__restrict__ v, double *__restrict__ lmax) {
    const double nrm = sqrt(dots[0]);
    const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) lmax[0] = nrm > 0.0 ? nrm : 1.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = w[i] * inv;
}

// dense coarsest matrix from the block pattern
template <int B, typename V = double>
__global__ void k_bsr_to_dense(int64_t nrows, const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                               const V *__restrict__ A, int64_t N, double *__restrict__ D) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nrows; i += (int64_t)gridDim.x * blockDim.x)
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            const int64_t j = col[p];
#pragma unroll
            for (int a = 0; a < B; ++a)
#pragma unroll
                for (int b = 0; b < B; ++b) D[(i * B + a) * N + j * B + b] = A[(int64_t)p * B * B + a * B + b];
        }
}

// Gauss-Jordan inversion (SPD, no pivoting), pivot k: save column k and the scaled row k
__global__ void k_gj_save(int64_t N, int64_t k, const double *__restrict__ D, double *__restrict__ colk,
                          double *__restrict__ rowk) {
    const double piv = D[k * N + k];
    const double ip = piv != 0.0 ? 1.0 / piv : 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < N; t += (int64_t)gridDim.x * blockDim.x) {
        colk[t] = D[t * N + k];
        rowk[t] = D[k * N + t] * ip;
    }
}
__global__ void k_gj_update(int64_t N, int64_t k, double *__restrict__ D, const double *__restrict__ colk,
                            const double *__restrict__ rowk) {
    const double piv = colk[k];
    const double ip = piv != 0.0 ? 1.0 / piv : 0.0;
    const int64_t total = N * N;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / N, j = t - i * N;
        double v;
        if (i == k && j == k) v = ip;
        else if (i == k) v = rowk[j];
        else if (j == k) v = -colk[i] * ip;
        else v = D[t] - colk[i] * rowk[j];
        D[t] = v;
    }
}

// Blocked Gauss-Jordan inversion (SPD, no pivoting) with NB x NB pivot blocks:
//   1. k_gjb_pivot : invert the pivot block in shared memory (one CTA) -> Pinv
//   2. k_gjb_save  : keep the pivot column block C = D(:, K) and the scaled row block
//                    Rw = Pinv D(K, :)
//   3. k_gjb_update: D(K,K) = Pinv, D(K,j) = Rw(:,j), D(i,K) = -C(i,:) Pinv,
//                    D(i,j) -= C(i,:) Rw(:,j)
constexpr int GJ_NB = 32;

__global__ void __launch_bounds__(GJ_NB * GJ_NB) k_gjb_pivot(int64_t N, int64_t k0, int nb, const double *__restrict__ D,
                                                             double *__restrict__ Pinv) {
    __shared__ double m[GJ_NB][2 * GJ_NB + 1];
    const int r = threadIdx.x / GJ_NB, c = threadIdx.x % GJ_NB;
    if (r < nb && c < nb) {
        m[r][c] = D[(k0 + r) * N + k0 + c];
        m[r][GJ_NB + c] = (r == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int k = 0; k < nb; ++k) {
        // every thread owns entries (r, c) and (r, c + NB); all reads happen before the barrier,
        // all writes after it
        double n0 = 0.0, n1 = 0.0;
        if (r < nb) {
            const double piv = m[k][k];
            const double ip = piv != 0.0 ? 1.0 / piv : 0.0;
            const double fk = m[r][k];
            const double rk0 = m[k][c] * ip, rk1 = m[k][c + GJ_NB] * ip;
            n0 = (r == k) ? rk0 : m[r][c] - fk * rk0;
            n1 = (r == k) ? rk1 : m[r][c + GJ_NB] - fk * rk1;
        }
        __syncthreads();
        if (r < nb) {
            m[r][c] = n0;
            m[r][c + GJ_NB] = n1;
        }
        __syncthreads();
    }
    if (r < nb && c < nb) Pinv[r * GJ_NB + c] = m[r][GJ_NB + c];
}

__global__ void k_gjb_save(int64_t N, int64_t k0, int nb, const double *__restrict__ D,
                           const double *__restrict__ Pinv, double *__restrict__ C, double *__restrict__ Rw) {
    const int64_t total = N * nb;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / nb;
        const int c = (int)(t - i * nb);
        C[i * GJ_NB + c] = D[i * N + k0 + c];                // column block
        double s = 0.0;                                      // Rw(c, j = i) = sum_m Pinv(c, m) D(k0 + m, i)
        for (int m = 0; m < nb; ++m) s += Pinv[c * GJ_NB + m] * D[(k0 + m) * N + i];
        Rw[c * N + i] = s;
    }
}

__global__ void k_gjb_update(int64_t N, int64_t k0, int nb, double *__restrict__ D, const double *__restrict__ Pinv,
                             const double *__restrict__ C, const double *__restrict__ Rw) {
    const int64_t total = N * N;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / N, j = t - i * N;
        const bool ik = (i >= k0 && i < k0 + nb), jk = (j >= k0 && j < k0 + nb);
        double v;
        if (ik && jk) {
            v = Pinv[(i - k0) * GJ_NB + (j - k0)];
        } else if (ik) {
            v = Rw[(i - k0) * N + j];
        } else if (jk) {
            double s = 0.0;
            for (int m = 0; m < nb; ++m) s += C[i * GJ_NB + m] * Pinv[m * GJ_NB + (j - k0)];
            v = -s;
        } else {
            double s = 0.0;
            for (int m = 0; m < nb; ++m) s += C[i * GJ_NB + m] * Rw[m * N + j];
            v = D[t] - s;
        }
        D[t] = v;
    }
}

template <typename T>
__global__ void k_dense_gemv(int64_t N, const T *__restrict__ M, const T *__restrict__ x, T *__restrict__ y) {
    // one warp per row
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < N; i += nw) {
        T s = 0;
        for (int64_t j = lane; j < N; j += 32) s += M[i * N + j] * x[j];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) y[i] = s;
    }
}

// ------------------------------------------------------------------ dispatch helpers

#define SG_B_DISPATCH(bval, BODY)                                 \
    switch (bval) {                                               \
        case 1: { constexpr int BB = 1; BODY; } break;            \
        case 2: { constexpr int BB = 2; BODY; } break;            \
        case 3: { constexpr int BB = 3; BODY; } break;            \
        case 6: { constexpr int BB = 6; BODY; } break;            \
        default: return set_error(SG_ERR_ARG, "AMG block size must be 1, 2, 3 or 6"); \
    }

#define SG_BBC_DISPATCH(bv, bcv, BODY)                                            \
    if (bv == 3 && bcv == 6) { constexpr int BB = 3, BC = 6; BODY; }              \
    else if (bv == 6 && bcv == 6) { constexpr int BB = 6, BC = 6; BODY; }         \
    else if (bv == 2 && bcv == 3) { constexpr int BB = 2, BC = 3; BODY; }         \
    else if (bv == 3 && bcv == 3) { constexpr int BB = 3, BC = 3; BODY; }         \
    else if (bv == 1 && bcv == 1) { constexpr int BB = 1, BC = 1; BODY; }         \
    else return set_error(SG_ERR_ARG, "unsupported AMG block shape");

static int free_level(Level &l) {
    auto F = [](void *p) { if (p) cudaFree(p); };
    F(l.Aown.d_rp); F(l.Aown.d_col); F(l.d_diag_own); F(l.Aown_vals); F(l.A32); F(l.A16); F(l.Dinv); F(l.Dinv32);
    F(l.lmax); F(l.d_dead); F(l.d_agg); F(l.T); F(l.P.d_rp); F(l.P.d_col); F(l.R.d_rp); F(l.R.d_col);
    F(l.AP.d_rp); F(l.AP.d_col); F(l.d_R_from_P); F(l.d_ac_out); F(l.d_ac_lower); F(l.d_ac_lower_src);
    F(l.Aown.d_row); F(l.P.d_row); F(l.R.d_row); F(l.AP.d_row);
    for (Plan *p : {&l.at_plan, &l.ap_plan, &l.ac_plan}) { F(p->d_ptr); F(p->d_a); F(p->d_b); }
    F(l.Pv); F(l.Rv); F(l.APv); F(l.P32); F(l.R32); F(l.T32); F(l.APv32);
    F(l.x); F(l.rhs); F(l.r); F(l.d); F(l.t); F(l.pv); F(l.x32); F(l.rhs32); F(l.r32); F(l.d32);
    return SG_OK;
}

static int alloc_level_buffers(Level &L, int mixed) {
    const size_t nb = (size_t)L.n * L.b;
    int rc = dalloc(&L.Dinv, nb * L.b);
    if (!rc) rc = dalloc(&L.lmax, 4);
    if (!rc) rc = dalloc(&L.x, nb);
    if (!rc) rc = dalloc(&L.rhs, nb);
    if (!rc) rc = dalloc(&L.r, nb);
    if (!rc) rc = dalloc(&L.d, nb);
    if (!rc) rc = dalloc(&L.pv, nb);
    if (!rc) rc = dalloc(&L.t, nb);
    if (!rc && mixed) {
        rc = dalloc(&L.Dinv32, nb * L.b);
        if (!rc) rc = dalloc(&L.A32, (size_t)L.Anblk * L.b * L.b);
        if (!rc) rc = dalloc(&L.x32, nb);
        if (!rc) rc = dalloc(&L.rhs32, nb);
        if (!rc) rc = dalloc(&L.r32, nb);
        if (!rc) rc = dalloc(&L.d32, nb);
    }
    return rc;
}

// Structure of the transfer from level L (pattern rp/col, near-null space B) to the next
// level.  Returns the coarse pattern, coarse near-null space and dead-DOF flags.
static int setup_transfer(Level &L, const std::vector<int32_t> &rp, const std::vector<int32_t> &col,
                          const std::vector<double> &B, int nns, int64_t na, Pattern &Ac, std::vector<double> &Bc,
                          std::vector<uint8_t> &dead, int mixed, int symmetric) {
    const int64_t n = L.n;
    const int b = L.b, bc = nns;
    L.bc = bc;
    std::vector<double> T;
    tentative(n, b, nns, na, L.agg, B, T, Bc, dead);
    // P pattern + plan for A T: P block (i, J) <- A blocks (i, k) with agg(k) == J
    build_product(n, L.P, L.at_plan, [&](int64_t i, std::vector<std::array<int32_t, 3>> &tr) {
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            const int32_t a = L.agg[col[p]];
            if (a >= 0) tr.push_back({a, p, 0});
        }
    });
    L.P.ncols = na;
    // R = P' pattern and the block map
    Pattern &R = L.R;
    R.nrows = na;
    R.ncols = n;
    R.rp.assign(na + 1, 0);
    for (int32_t c : L.P.col) R.rp[c + 1]++;
    for (int64_t I = 0; I < na; ++I) R.rp[I + 1] += R.rp[I];
    R.nblk = L.P.nblk;
    R.col.resize(R.nblk);
    std::vector<int32_t> fill(R.rp.begin(), R.rp.end() - 1), from(R.nblk), pblk_of_r(R.nblk);
    for (int64_t i = 0; i < n; ++i)
        for (int32_t q = L.P.rp[i]; q < L.P.rp[i + 1]; ++q) {
            const int32_t I = L.P.col[q];
            R.col[fill[I]] = (int32_t)i;
            from[fill[I]++] = q;
        }
    // AP pattern + plan: (i, J) <- pairs (A block (i, k), P block (k, J)).  With a symmetric A
    // only the coarse blocks (I, J), I <= J, are formed, and AP(i, J) enters them only through
    // P(i, I)' AP(i, J) with I <= J: blocks with J below the smallest coarse column of P's row
    // i are never read and are left out.
    std::vector<int32_t> lo_col(n, 0);
    if (symmetric)
        for (int64_t i = 0; i < n; ++i)
            lo_col[i] = L.P.rp[i] < L.P.rp[i + 1] ? L.P.col[L.P.rp[i]] : INT32_MAX;
    build_product(n, L.AP, L.ap_plan, [&](int64_t i, std::vector<std::array<int32_t, 3>> &tr) {
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            const int32_t k = col[p];
            for (int32_t q = L.P.rp[k]; q < L.P.rp[k + 1]; ++q)
                if (L.P.col[q] >= lo_col[i]) tr.push_back({L.P.col[q], p, q});
        }
    });
    L.AP.ncols = na;
    // Ac pattern + plan: (I, J) <- pairs (P block (i, I), AP block (i, J))
    auto ac_pairs_of = [&](bool upper) {
        return [&, upper](int64_t I, std::vector<std::array<int32_t, 3>> &tr) {
            for (int32_t k = R.rp[I]; k < R.rp[I + 1]; ++k) {
                const int32_t i = R.col[k];
                const int32_t pblk = from[k];
                for (int32_t q = L.AP.rp[i]; q < L.AP.rp[i + 1]; ++q)
                    if (!upper || L.AP.col[q] >= I) tr.push_back({L.AP.col[q], pblk, q});
            }
        };
    };
    std::vector<int32_t> ac_out, ac_lower, ac_lower_src;
    if (!symmetric) {
        build_product(na, Ac, L.ac_plan, ac_pairs_of(false));
    } else {
        // plan over the upper blocks U (I <= J); the coarse pattern is U and its transpose:
        // row I holds the columns J < I of the mirrored blocks, then U's row I
        Pattern U;
        build_product(na, U, L.ac_plan, ac_pairs_of(true));
        std::vector<std::vector<int32_t>> low(na);
        for (int64_t J = 0; J < na; ++J)
            for (int32_t u = U.rp[J]; u < U.rp[J + 1]; ++u)
                if (U.col[u] > J) low[U.col[u]].push_back((int32_t)J);
        Ac.nrows = na;
        Ac.rp.assign(na + 1, 0);
        for (int64_t I = 0; I < na; ++I)
            Ac.rp[I + 1] = Ac.rp[I] + (int32_t)low[I].size() + (U.rp[I + 1] - U.rp[I]);
        Ac.nblk = Ac.rp[na];
        Ac.col.resize(Ac.nblk);
        ac_out.resize(U.nblk);
        for (int64_t I = 0; I < na; ++I) {
            int32_t o = Ac.rp[I];
            for (int32_t J : low[I]) Ac.col[o++] = J;
            for (int32_t u = U.rp[I]; u < U.rp[I + 1]; ++u) {
                ac_out[u] = o;
                Ac.col[o++] = U.col[u];
            }
        }
        for (int64_t I = 0; I < na; ++I)
            for (size_t m = 0; m < low[I].size(); ++m) {
                const int32_t J = low[I][m];
                const int32_t *b0 = U.col.data() + U.rp[J], *b1 = U.col.data() + U.rp[J + 1];
                const int32_t u = (int32_t)(std::lower_bound(b0, b1, (int32_t)I) - U.col.data());
                ac_lower.push_back(Ac.rp[I] + (int32_t)m);
                ac_lower_src.push_back(ac_out[u]);
            }
        L.n_ac_items = U.nblk;
        L.n_ac_lower = (int64_t)ac_lower.size();
    }
    Ac.ncols = na;
    int rc = dup(&L.d_R_from_P, from);
    if (!rc && symmetric) rc = dup(&L.d_ac_out, ac_out);
    if (!rc && symmetric) rc = dup(&L.d_ac_lower, ac_lower);
    if (!rc && symmetric) rc = dup(&L.d_ac_lower_src, ac_lower_src);
    if (!rc) rc = dup(&L.d_agg, L.agg);
    if (!rc) rc = dup(&L.T, T);
    if (!rc) rc = upload_pattern(L.P);
    if (!rc) rc = upload_pattern(L.R);
    if (!rc) rc = upload_pattern(L.AP);
    if (!rc) rc = upload_plan(L.at_plan);
    if (!rc) rc = upload_plan(L.ap_plan);
    if (!rc) rc = upload_plan(L.ac_plan);
    if (!rc) rc = dalloc(&L.Pv, (size_t)L.P.nblk * b * bc);
    if (!rc) rc = dalloc(&L.Rv, (size_t)L.P.nblk * b * bc);
    if (!rc) rc = dalloc(&L.APv, (size_t)L.AP.nblk * b * bc);
    if (!rc && mixed) rc = dalloc(&L.P32, (size_t)L.P.nblk * b * bc);
    if (!rc && mixed) rc = dalloc(&L.R32, (size_t)L.P.nblk * b * bc);
    if (!rc && mixed) rc = dalloc(&L.APv32, (size_t)L.AP.nblk * b * bc);
    if (!rc && mixed) {
        std::vector<float> t32(T.begin(), T.end());
        rc = dup(&L.T32, t32);
    }
    L.ap_pairs = (int64_t)L.ap_plan.a.size();
    L.ac_pairs = (int64_t)L.ac_plan.a.size();
    for (Plan *pl : {&L.at_plan, &L.ap_plan, &L.ac_plan}) {  // host copies no longer needed
        std::vector<int64_t>().swap(pl->ptr);
        std::vector<int32_t>().swap(pl->a);
        std::vector<int32_t>().swap(pl->b);
    }
    return rc;
}

// ------------------------------------------------------------------ numeric set-up

static const double *level_values(const Level &L) { return L.Aext ? L.Avals : L.Aown_vals; }

static int power_lmax(sg_amg *h, Level &L, const double *A, cudaStream_t st) {
    const int64_t nd = L.n * L.b;
    // cold (deterministic start vector, power_its steps) for the set-up inside sg_amg_create and
    // for the first sg_amg_update, warm afterwards
    const bool warm = L.power_warm >= 2;
    if (!warm) k_init_vec<<<grid_for(nd, 256), 256, 0, st>>>(nd, L.pv);
    ++L.power_warm;
    int rc = SG_OK;
    const int its = warm ? h->opt.power_its_warm : h->opt.power_its;
    for (int it = 0; it < its && !rc; ++it) {
        rc = rect_spmv<double, double>(L.b, L.b, L.n, L.d_Arp, L.d_Acol, A, L.pv, L.t, 1.0, 0.0, nullptr, 0, st, L.Anblk);
        if (rc) break;
        SG_B_DISPATCH(L.b, (k_dinv_apply<BB, double><<<grid_for(L.n, 256), 256, 0, st>>>(L.n, L.Dinv, L.t, L.r)));
        rc = multidot(nd, 1, L.r, nd, L.r, h->dots, h->dots + DOT_BLOCKS, st);
        if (rc) break;
        k_power_norm<<<grid_for(nd, 256), 256, 0, st>>>(nd, L.r, h->dots + DOT_BLOCKS, L.pv, L.lmax);
    }
    SG_CUDA(cudaGetLastError());
    return rc;
}

// lambda_max of D^-1 A from the FP32 level matrix (FP64 vectors), same start and step rules.
static int power_lmax32(sg_amg *h, Level &L, cudaStream_t st) {
    const int64_t nd = L.n * L.b;
    const bool warm = L.power_warm >= 2;
    if (!warm) k_init_vec<<<grid_for(nd, 256), 256, 0, st>>>(nd, L.pv);
    ++L.power_warm;
    int rc = SG_OK;
    const int its = warm ? h->opt.power_its_warm : h->opt.power_its;
    for (int it = 0; it < its && !rc; ++it) {
        rc = rect_spmv<float, double>(L.b, L.b, L.n, L.d_Arp, L.d_Acol, L.A32, L.pv, L.t, 1.0, 0.0, nullptr, 0, st,
                                      L.Anblk);
        if (rc) break;
        SG_B_DISPATCH(L.b, (k_dinv_apply<BB, double><<<grid_for(L.n, 256), 256, 0, st>>>(L.n, L.Dinv, L.t, L.r)));
        rc = multidot(nd, 1, L.r, nd, L.r, h->dots, h->dots + DOT_BLOCKS, st);
        if (rc) break;
        k_power_norm<<<grid_for(nd, 256), 256, 0, st>>>(nd, L.r, h->dots + DOT_BLOCKS, L.pv, L.lmax);
    }
    SG_CUDA(cudaGetLastError());
    return rc;
}

// Block-Jacobi inverse of level l (and the FP32 copy of its matrix).
static int numeric_smoother(sg_amg *h, int l, cudaStream_t st) {
    Level &L = h->L[l];
    const double *A = level_values(L);
    SG_B_DISPATCH(L.b, (k_block_diag_inv<BB><<<grid_for(L.n, 128), 128, 0, st>>>(L.n, L.d_Adiag, A, L.Dinv, L.Dinv32)));
    SG_CUDA(cudaGetLastError());
    if (h->opt.mixed) {
        const int64_t nv = L.Anblk * L.b * L.b;
        k_to_float<<<grid_for(nv, 256), 256, 0, st>>>(nv, A, L.A32);
    }
    return SG_OK;
}

// lambda_max, prolongator, restriction and the next level's Galerkin matrix.
static int numeric_transfer(sg_amg *h, int l, cudaStream_t st) {
    Level &L = h->L[l];
    Level &C = h->L[l + 1];
    const double *A = level_values(L);
    int rc = power_lmax(h, L, A, st);
    if (rc) return rc;
    SG_BBC_DISPATCH(L.b, L.bc, ({
        const int64_t pch = chunk_len(L.P.nblk, 128, 8 * 128);
        k_smooth_prolongator<BB, BC><<<grid_chunks(L.P.nblk, pch), 128, 0, st>>>(
            L.P.nblk, L.P.d_row, L.P.d_col, L.at_plan.d_ptr, L.at_plan.d_a, L.d_Acol, A, L.T, L.d_agg, L.Dinv, L.lmax,
            h->opt.omega_scale, L.Pv, pch);
        k_transpose_blocks<BB, BC><<<grid_for(L.P.nblk * BB * BC, 256), 256, 0, st>>>(L.P.nblk, L.d_R_from_P, L.Pv, L.Rv);
        // one thread per output block, or a warp per block where blocks are few or each sums
        // many pairs (measured on the SSR hierarchy: fine-level A P, ~15 pairs per block, is
        // faster per thread; P'(A P), ~63 pairs per block, 1.3x faster per warp; the small
        // coarse levels 10-20x faster per warp)
        auto per_warp = [](int64_t nblk, int64_t pairs) { return nblk < 32768 || pairs >= 24 * nblk; };
        if (!per_warp(L.AP.nblk, L.ap_pairs)) {
            const int64_t ach = chunk_len(L.AP.nblk, 128, 8 * 128);
            k_gather_AP<BB, BC><<<grid_chunks(L.AP.nblk, ach), 128, 0, st>>>(L.AP.nblk, L.ap_plan.d_ptr,
                                                                             L.ap_plan.d_a, L.ap_plan.d_b, A, L.Pv,
                                                                             L.APv, ach);
        } else
            gather_AP_groups<BB, BC, double>(L.AP.nblk, L.ap_pairs, L.ap_plan.d_ptr, L.ap_plan.d_a, L.ap_plan.d_b, A,
                                             L.Pv, L.APv, st);
        galerkin_Ac<BB, BC, double>(L, C, L.Pv, L.APv, C.Aown_vals, st);
    }));
    SG_CUDA(cudaGetLastError());
    if (h->opt.mixed) {
        const int64_t np_ = L.P.nblk * L.b * L.bc;
        k_to_float<<<grid_for(np_, 256), 256, 0, st>>>(np_, L.Pv, L.P32);
        k_to_float<<<grid_for(np_, 256), 256, 0, st>>>(np_, L.Rv, L.R32);
    }
    return SG_OK;
}

static int numeric_coarsest(sg_amg *h, cudaStream_t st) {
    Level &L = h->L.back();
    const double *A = level_values(L);
    const int64_t N = h->nc_dense;
    SG_CUDA(cudaMemsetAsync(h->Ainv, 0, sizeof(double) * N * N, st));
    SG_B_DISPATCH(L.b, (k_bsr_to_dense<BB><<<grid_for(L.n, 128), 128, 0, st>>>(L.n, L.d_Arp, L.d_Acol, A, N, h->Ainv)));
    for (int64_t k0 = 0; k0 < N; k0 += GJ_NB) {
        const int nb = (int)std::min<int64_t>(GJ_NB, N - k0);
        count_launch();
        k_gjb_pivot<<<1, GJ_NB * GJ_NB, 0, st>>>(N, k0, nb, h->Ainv, h->gj_pinv);
        k_gjb_save<<<grid_for(N * nb, 256), 256, 0, st>>>(N, k0, nb, h->Ainv, h->gj_pinv, h->colk, h->rowk);
        k_gjb_update<<<grid_for(N * N, 256, 16), 256, 0, st>>>(N, k0, nb, h->Ainv, h->gj_pinv, h->colk, h->rowk);
    }
    if (h->opt.mixed) k_to_float<<<grid_for(N * N, 256), 256, 0, st>>>(N * N, h->Ainv, h->Ainv32);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

static int numeric_update(sg_amg *h, cudaStream_t st) {
    const int nl = (int)h->L.size();
    int rc = SG_OK;
    for (int l = 0; l < nl && !rc; ++l) {
        rc = numeric_smoother(h, l, st);
        if (rc) break;
        rc = (l == nl - 1) ? numeric_coarsest(h, st) : numeric_transfer(h, l, st);
    }
    return rc;
}

// Mixed form: the numeric update in FP32 for the FP32 V-cycle.  The level matrices, P, R and
// A P are formed directly in FP32 (the Galerkin gathers accumulate in FP32, the prolongator
// smoothing in FP64 registers), the block inverses and lambda_max in FP64 from the FP32
// values; the coarsest dense inverse in FP64.
// The set-up inside sg_amg_create keeps the FP64 path, so the mixed form has the same
// hierarchy structure as the plain one.
static int numeric_update32(sg_amg *h, cudaStream_t st) {
    const int nl = (int)h->L.size();
    for (int l = 0; l < nl; ++l) {
        Level &L = h->L[l];
        if (l == 0) {
            const int64_t nv = L.Anblk * L.b * L.b;
            if (L.A16) {
                const int rc0 = to_float_half3(L.Anblk, L.Avals, L.A32, L.A16, L.a16_scale, st);
                if (rc0) return rc0;
            } else {
                k_to_float<<<grid_for(nv, 256), 256, 0, st>>>(nv, L.Avals, L.A32);
            }
        }
        SG_B_DISPATCH(L.b, (k_block_diag_inv<BB, float><<<grid_for(L.n, 128), 128, 0, st>>>(L.n, L.d_Adiag, L.A32,
                                                                                            L.Dinv, L.Dinv32)));
        SG_CUDA(cudaGetLastError());
        if (l == nl - 1) {
            const int64_t N = h->nc_dense;
            SG_CUDA(cudaMemsetAsync(h->Ainv, 0, sizeof(double) * N * N, st));
            SG_B_DISPATCH(L.b, (k_bsr_to_dense<BB, float><<<grid_for(L.n, 128), 128, 0, st>>>(
                                   L.n, L.d_Arp, L.d_Acol, L.A32, N, h->Ainv)));
            for (int64_t k0 = 0; k0 < N; k0 += GJ_NB) {
                const int nb = (int)std::min<int64_t>(GJ_NB, N - k0);
                count_launch();
                k_gjb_pivot<<<1, GJ_NB * GJ_NB, 0, st>>>(N, k0, nb, h->Ainv, h->gj_pinv);
                k_gjb_save<<<grid_for(N * nb, 256), 256, 0, st>>>(N, k0, nb, h->Ainv, h->gj_pinv, h->colk, h->rowk);
                k_gjb_update<<<grid_for(N * N, 256, 16), 256, 0, st>>>(N, k0, nb, h->Ainv, h->gj_pinv, h->colk,
                                                                      h->rowk);
            }
            k_to_float<<<grid_for(N * N, 256), 256, 0, st>>>(N * N, h->Ainv, h->Ainv32);
            SG_CUDA(cudaGetLastError());
            break;
        }
        Level &C = h->L[l + 1];
        int rc = power_lmax32(h, L, st);
        if (rc) return rc;
        SG_BBC_DISPATCH(L.b, L.bc, ({
            const int64_t pch = chunk_len(L.P.nblk, 128, 8 * 128);
            k_smooth_prolongator<BB, BC, float><<<grid_chunks(L.P.nblk, pch), 128, 0, st>>>(
                L.P.nblk, L.P.d_row, L.P.d_col, L.at_plan.d_ptr, L.at_plan.d_a, L.d_Acol, L.A32, L.T32, L.d_agg,
                L.Dinv, L.lmax, h->opt.omega_scale, L.P32, pch);
            k_transpose_blocks<BB, BC, float><<<grid_for(L.P.nblk * BB * BC, 256), 256, 0, st>>>(
                L.P.nblk, L.d_R_from_P, L.P32, L.R32);
            auto per_warp = [](int64_t nblk, int64_t pairs) { return nblk < 32768 || pairs >= 24 * nblk; };
            if (!per_warp(L.AP.nblk, L.ap_pairs)) {
                const int64_t ach = chunk_len(L.AP.nblk, 128, 8 * 128);
                k_gather_AP<BB, BC, float><<<grid_chunks(L.AP.nblk, ach), 128, 0, st>>>(
                    L.AP.nblk, L.ap_plan.d_ptr, L.ap_plan.d_a, L.ap_plan.d_b, L.A32, L.P32, L.APv32, ach);
            } else
                gather_AP_groups<BB, BC, float>(L.AP.nblk, L.ap_pairs, L.ap_plan.d_ptr, L.ap_plan.d_a, L.ap_plan.d_b,
                                                L.A32, L.P32, L.APv32, st);
            galerkin_Ac<BB, BC, float>(L, C, L.P32, L.APv32, C.A32, st);
        }));
        SG_CUDA(cudaGetLastError());
    }
    return SG_OK;
}

// ------------------------------------------------------------------ hierarchy structure

// Strength graph: keep block (i, j) when ||A_ij||_F >= theta sqrt(||A_ii||_F ||A_jj||_F), and i == j.
static void strength_graph(int64_t n, int b, const std::vector<int32_t> &rp, const std::vector<int32_t> &col,
                           const std::vector<double> &vals, double theta, std::vector<int32_t> &srp,
                           std::vector<int32_t> &scol) {
    const int64_t nb = rp[n];
    std::vector<double> nrm(nb), dg(n, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < nb; ++p) {
        double s = 0.0;
        for (int t = 0; t < b * b; ++t) s += vals[(size_t)p * b * b + t] * vals[(size_t)p * b * b + t];
        nrm[p] = std::sqrt(s);
    }
    for (int64_t i = 0; i < n; ++i)
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p)
            if (col[p] == i) dg[i] = nrm[p];
    srp.assign(n + 1, 0);
    scol.clear();
    scol.reserve(nb);
    for (int64_t i = 0; i < n; ++i) {
        for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
            const int32_t j = col[p];
            if (j == i || nrm[p] >= theta * std::sqrt(dg[i] * dg[j])) scol.push_back(j);
        }
        srp[i + 1] = (int32_t)scol.size();
    }
}

static int make_level(sg_amg *h, const sg_bsr *A0, const std::vector<int32_t> &rp, const std::vector<int32_t> &col,
                      int b, int64_t n, const std::vector<uint8_t> &dead) {
    h->L.emplace_back();
    Level &L = h->L.back();
    L.b = b;
    L.n = n;
    int rc = SG_OK;
    if (A0) {
        L.Aext = A0;
        L.d_Arp = A0->d_row_ptr;
        L.d_Acol = A0->d_col;
        L.d_Adiag = A0->d_diag;
        L.Anblk = A0->n_blocks;
    } else {
        L.Aown.nrows = n;
        L.Aown.ncols = n;
        L.Aown.rp = rp;
        L.Aown.col = col;
        L.Aown.nblk = rp[n];
        rc = upload_pattern(L.Aown);
        std::vector<int32_t> diag(n, -1);
        for (int64_t i = 0; i < n; ++i)
            for (int32_t p = rp[i]; p < rp[i + 1]; ++p)
                if (col[p] == i) diag[i] = p;
        if (!rc) rc = dup(&L.d_diag_own, diag);
        if (!rc) rc = dalloc(&L.Aown_vals, (size_t)L.Aown.nblk * b * b);
        if (!rc) rc = dup(&L.d_dead, dead);
        L.d_Arp = L.Aown.d_rp;
        L.d_Acol = L.Aown.d_col;
        L.d_Adiag = L.d_diag_own;
        L.Anblk = L.Aown.nblk;
    }
    if (!rc) rc = alloc_level_buffers(L, h->opt.mixed);
    return rc;
}

// Builds the hierarchy structure.  With A0vals (device values of the fine matrix) and
// theta > 0, every level's aggregation runs on its strength graph; the numeric set-up of a
// level is then done as soon as its transfer exists, so the next level's values are known.
static int build_hierarchy(sg_amg *h, const sg_bsr *A0, const double *A0vals, const double *nullspace, int nns,
                           const uint8_t *fixed, cudaStream_t st) {
    const AmgOptions &o = h->opt;
    h->L.reserve(o.max_levels + 2);
    std::vector<int32_t> rp = A0->row_ptr, col = A0->col;
    int b = A0->b;
    int64_t n = A0->n_rows;
    std::vector<double> B((size_t)n * b * nns);
    std::vector<uint8_t> active(n, 0), dead;
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < b; ++a) {
            const int64_t row = i * b + a;
            const bool fx = fixed && fixed[row];
            for (int c = 0; c < nns; ++c) B[(size_t)row * nns + c] = fx ? 0.0 : nullspace[(size_t)c * n * b + row];
            if (!fx) active[i] = 1;
        }
    const bool with_values = A0vals != nullptr && o.theta > 0.0;
    int rc = make_level(h, A0, rp, col, b, n, dead);
    if (rc) return rc;
    if (A0vals) h->L[0].Avals = A0vals;
    for (int lev = 0;; ++lev) {
        Level &L = h->L[lev];
        const int64_t ndof = n * b;
        const bool last = (ndof <= o.coarse_size) || (lev + 1 >= o.max_levels);
        int64_t na = 0;
        if (!last) {
            if (with_values) {
                std::vector<double> vals((size_t)rp[n] * b * b);
                SG_CUDA(cudaMemcpyAsync(vals.data(), level_values(L), sizeof(double) * vals.size(),
                                        cudaMemcpyDeviceToHost, st));
                SG_CUDA(cudaStreamSynchronize(st));
                if (lev == 0 && o.mixed && o.fine_half && b == 3) {
                    // FP16 copy of level 0: a power-of-two scale maps the largest entry of the
                    // set-up matrix to (2048, 4096], leaving 16x headroom below the FP16 maximum
                    // for later value updates (larger magnitudes are clamped)
                    double mx = 0.0;
                    for (double v : vals) mx = std::max(mx, std::fabs(v));
                    if (mx > 0.0 && std::isfinite(mx)) {
                        L.a16_scale = (float)std::ldexp(1.0, (int)std::ceil(std::log2(mx / 4096.0)));
                        rc = dalloc(&L.A16, (size_t)L.Anblk * 3);
                        if (rc) return rc;
                    }
                }
                std::vector<int32_t> srp, scol;
                strength_graph(n, b, rp, col, vals, o.theta, srp, scol);
                na = aggregate(n, srp, scol, active, L.agg);
            } else {
                na = aggregate(n, rp, col, active, L.agg);
            }
        }
        if (last || na == 0 || na * nns >= ndof * 3 / 4) {
            std::vector<int32_t>().swap(L.agg);
            if (ndof > 12000)
                return set_error(SG_ERR_NUMERIC, "AMG coarsening stalled: coarsest level too large for a dense inverse");
            h->nc_dense = ndof;
            rc = dalloc(&h->Ainv, (size_t)ndof * ndof);
            if (!rc) rc = dalloc(&h->colk, (size_t)ndof * GJ_NB);
            if (!rc) rc = dalloc(&h->rowk, (size_t)ndof * GJ_NB);
            if (!rc) rc = dalloc(&h->gj_pinv, (size_t)GJ_NB * GJ_NB);
            if (!rc && o.mixed) rc = dalloc(&h->Ainv32, (size_t)ndof * ndof);
            return rc;
        }
        Pattern Ac;
        std::vector<double> Bc;
        std::vector<uint8_t> dead_c;
        rc = setup_transfer(L, rp, col, B, nns, na, Ac, Bc, dead_c, o.mixed, o.symmetric);
        if (rc) return rc;
        rc = make_level(h, nullptr, Ac.rp, Ac.col, nns, na, dead_c);
        if (rc) return rc;
        if (with_values) {
            rc = numeric_smoother(h, lev, st);
            if (!rc) rc = numeric_transfer(h, lev, st);
            if (rc) return rc;
        }
        rp = std::move(Ac.rp);
        col = std::move(Ac.col);
        b = nns;
        n = na;
        B = std::move(Bc);
        dead = std::move(dead_c);
        active.assign(n, 0);
        for (int64_t i = 0; i < n; ++i)
            for (int c = 0; c < b; ++c) active[i] |= !dead[(size_t)i * b + c];
    }
}

// x_i += C_i r_i for 3 x 3 node blocks C (row-major)
template <typename T>
__global__ void k_corr_apply(int64_t n, const T *__restrict__ Cb, const T *__restrict__ r, T *__restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T *c = Cb + i * 9;
        const T r0 = r[3 * i], r1 = r[3 * i + 1], r2 = r[3 * i + 2];
        x[3 * i] += c[0] * r0 + c[1] * r1 + c[2] * r2;
        x[3 * i + 1] += c[3] * r0 + c[4] * r1 + c[5] * r2;
        x[3 * i + 2] += c[6] * r0 + c[7] * r1 + c[8] * r2;
    }
}

// ------------------------------------------------------------------ V-cycle

template <typename T>
struct LevelView {
    const T *A, *Dinv, *P, *R;
    T *x, *rhs, *r, *d;
};

template <typename T>
static LevelView<T> view(Level &L);
template <>
LevelView<double> view<double>(Level &L) {
    return {L.Aext ? L.Avals : L.Aown_vals, L.Dinv, L.Pv, L.Rv, L.x, L.rhs, L.r, L.d};
}
template <>
LevelView<float> view<float>(Level &L) {
    return {L.A32, L.Dinv32, L.P32, L.R32, L.x32, L.rhs32, L.r32, L.d32};
}

// r = rhs - A x on a level; level 0 of the FP32 cycle reads the FP16 copy when there is one
template <typename T>
static int level_residual(Level &L, LevelView<T> &v, cudaStream_t st) {
    if constexpr (std::is_same<T, float>::value) {
        if (L.A16) return h3_spmv(L.n, L.Anblk, L.d_Arp, L.d_Acol, L.A16, L.a16_scale, v.x, v.r, v.rhs, 1, st);
    }
    return rect_spmv<T, T>(L.b, L.b, L.n, L.d_Arp, L.d_Acol, v.A, v.x, v.r, 1.0, 0.0, v.rhs, 1, st, L.Anblk);
}

template <typename T>
static int smooth(sg_amg *h, Level &L, LevelView<T> &v, bool x_zero, cudaStream_t st) {
    const int deg = h->opt.cheb_degree;
    int rc = SG_OK;
    for (int k = 0; k < deg && !rc; ++k) {
        const T *r = v.rhs;
        if (!(x_zero && k == 0)) {
            rc = level_residual<T>(L, v, st);
            if (rc) return rc;
            r = v.r;
        }
        const int xz = (x_zero && k == 0) ? 1 : 0;
        SG_B_DISPATCH(L.b, (k_cheb<BB, T><<<grid_for(L.n, 256), 256, 0, st>>>(L.n, k, h->opt.cheb_ratio, L.lmax, v.Dinv, r, v.d, v.x, xz)));
    }
    SG_CUDA(cudaGetLastError());
    return rc;
}

template <typename T>
static int vcycle(sg_amg *h, int l, cudaStream_t st) {
    Level &L = h->L[l];
    LevelView<T> v = view<T>(L);
    if (l == (int)h->L.size() - 1) {
        const T *M = std::is_same<T, float>::value ? (const T *)h->Ainv32 : (const T *)h->Ainv;
        k_dense_gemv<T><<<grid_for(h->nc_dense * 32, 256), 256, 0, st>>>(h->nc_dense, M, v.rhs, v.x);
        SG_CUDA(cudaGetLastError());
        return SG_OK;
    }
    Level &C = h->L[l + 1];
    LevelView<T> c = view<T>(C);
    int rc = smooth<T>(h, L, v, true, st);
    if (!rc) rc = level_residual<T>(L, v, st);
    if (!rc) rc = rect_spmv<T, T>(L.bc, L.b, C.n, L.R.d_rp, L.R.d_col, v.R, v.r, c.rhs, 1.0, 0.0, nullptr, 0, st, L.R.nblk);
    if (!rc) rc = vcycle<T>(h, l + 1, st);
    if (!rc) rc = rect_spmv<T, T>(L.b, L.bc, L.n, L.P.d_rp, L.P.d_col, v.P, c.x, v.x, 1.0, 1.0, nullptr, 0, st, L.P.nblk);
    if (!rc) rc = smooth<T>(h, L, v, false, st);
    return rc;
}

}  // namespace sg

using namespace sg;

extern "C" int sg_amg_create(const sg_bsr *A, const double *A_vals, const double *nullspace, int32_t nns,
                             const uint8_t *fixed, const double *opts, int32_t n_opts, sg_amg **out,
                             void *stream) {
    SG_CHECK_ARG(out, "null output handle");
    *out = nullptr;
    SG_CHECK_ARG(A && nullspace, "null pattern or near-null space");
    SG_CHECK_ARG(nns > 0 && nns <= 6, "near-null space dimension must be 1..6");
    SG_CHECK_ARG((A->b == 3 && nns == 6) || (A->b == 2 && nns == 3) || (A->b == 3 && nns == 3) ||
                     (A->b == 1 && nns == 1),
                 "supported (block, near-null) sizes: (3,6), (3,3), (2,3), (1,1)");
    sg_amg *h = new (std::nothrow) sg_amg();
    if (!h) return set_error(SG_ERR_NOMEM, "host allocation");
    cudaGetDevice(&h->device);
    // opts: [max_levels, coarse_size, cheb_degree, cheb_ratio, power_its, mixed, omega_scale, theta,
    //        fine_half]
    if (opts) {
        if (n_opts > 0 && opts[0] > 0) h->opt.max_levels = (int)opts[0];
        if (n_opts > 1 && opts[1] > 0) h->opt.coarse_size = (int)opts[1];
        if (n_opts > 2 && opts[2] > 0) h->opt.cheb_degree = (int)opts[2];
        if (n_opts > 3 && opts[3] > 1) h->opt.cheb_ratio = opts[3];
        if (n_opts > 4 && opts[4] > 0) h->opt.power_its = (int)opts[4];
        if (n_opts > 5) h->opt.mixed = opts[5] != 0.0;
        if (n_opts > 6 && opts[6] > 0) h->opt.omega_scale = opts[6];
        if (n_opts > 7 && opts[7] >= 0) h->opt.theta = opts[7];
        if (n_opts > 8) h->opt.fine_half = opts[8] != 0.0;
        if (n_opts > 9) h->opt.symmetric = opts[9] != 0.0;
    }
    int rc = dalloc(&h->dots, DOT_BLOCKS + 64);
    if (!rc) rc = build_hierarchy(h, A, A_vals, nullspace, nns, fixed, as_stream(stream));
    if (rc) {
        for (auto &L : h->L) free_level(L);
        cudaFree(h->Ainv); cudaFree(h->Ainv32); cudaFree(h->colk); cudaFree(h->rowk); cudaFree(h->dots);
        cudaFree(h->gj_pinv);
        delete h;
        return rc;
    }
    *out = h;
    return SG_OK;
}

extern "C" int sg_amg_destroy(sg_amg *h) {
    if (!h) return SG_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(h->device);
    if (h->parent) {
        for (auto &L : h->L) {
            cudaFree(L.x); cudaFree(L.rhs); cudaFree(L.r); cudaFree(L.d);
            cudaFree(L.x32); cudaFree(L.rhs32); cudaFree(L.r32); cudaFree(L.d32);
        }
        cudaSetDevice(cur);
        delete h;
        return SG_OK;
    }
    for (auto &L : h->L) free_level(L);
    cudaFree(h->Ainv);
    cudaFree(h->Ainv32);
    cudaFree(h->colk);
    cudaFree(h->rowk);
    cudaFree(h->dots);
    cudaFree(h->gj_pinv);
    cudaFree(h->corrC);
    cudaFree(h->corrC32);
    cudaSetDevice(cur);
    delete h;
    return SG_OK;
}

// A second set of cycle vectors over the same hierarchy (no counterpart in the reference),
// so that two V-cycles can run at the same time on different streams (the two independent
// Krylov solves of a Newton step).  The clone reads the parent's matrices, transfer operators
// and inverses as the parent's updates leave them; only the parent is updated, the parent
// must outlive the clone, and the learned correction is not available on a clone.
extern "C" int sg_amg_clone(const sg_amg *h, sg_amg **out) {
    SG_CHECK_ARG(h && out, "null argument");
    SG_CHECK_ARG(!h->parent, "clone of a clone");
    *out = nullptr;
    sg_amg *c = new (std::nothrow) sg_amg(*h);
    if (!c) return set_error(SG_ERR_NOMEM, "host allocation");
    c->parent = h;
    c->corrC = nullptr;
    c->corrC32 = nullptr;
    c->corr_on = 0;
    int rc = SG_OK;
    for (auto &L : c->L) {
        L.x = L.rhs = L.r = L.d = nullptr;
        L.x32 = L.rhs32 = L.r32 = L.d32 = nullptr;
    }
    for (auto &L : c->L) {
        const size_t nb = (size_t)L.n * L.b;
        if (!rc) rc = dalloc(&L.x, nb);
        if (!rc) rc = dalloc(&L.rhs, nb);
        if (!rc) rc = dalloc(&L.r, nb);
        if (!rc) rc = dalloc(&L.d, nb);
        if (!rc && h->opt.mixed) {
            rc = dalloc(&L.x32, nb);
            if (!rc) rc = dalloc(&L.rhs32, nb);
            if (!rc) rc = dalloc(&L.r32, nb);
            if (!rc) rc = dalloc(&L.d32, nb);
        }
    }
    if (rc) {
        sg_amg_destroy(c);
        return rc;
    }
    *out = c;
    return SG_OK;
}

namespace sg {
// Everything a captured V-cycle (sg_amg_apply inside a CUDA graph) depends on beyond the
// hierarchy's own buffers: the level-0 values pointer (the caller's, in the FP64 cycle; the
// parent's for a clone) and whether the learned correction is on.  A graph that captured the
// cycle is valid while this key is unchanged.
uint64_t amg_capture_key(const sg_amg *h) {
    const double *a0 = h->parent ? h->parent->L[0].Avals : h->L[0].Avals;
    return (uint64_t)(uintptr_t)a0 * 31u + (uint64_t)(h->corr_on ? 1 : 0) + (uint64_t)(uintptr_t)h;
}
}  // namespace sg

// Numeric set-up for new values of the level-0 matrix (device pointer, kept by reference
// until the next update: the caller must not free or overwrite it while applying).
extern "C" int sg_amg_update(sg_amg *h, const double *Avals, void *stream) {
    SG_CHECK_ARG(h && Avals, "null argument");
    SG_CHECK_ARG(!h->parent, "a clone is updated through its parent");
    h->L[0].Avals = Avals;
    const InstrToken tk = instr_begin(IK_AMG_UPDATE, as_stream(stream));
    int rc = h->opt.mixed ? numeric_update32(h, as_stream(stream)) : numeric_update(h, as_stream(stream));
    instr_end(tk, as_stream(stream));
    if (!rc) h->updated = 1;
    return rc;
}

// z = one V-cycle applied to r (device pointers, FP64 in and out).
extern "C" int sg_amg_apply(sg_amg *h, const double *r, double *z, void *stream) {
    SG_CHECK_ARG(h && r && z, "null argument");
    if (h->parent) {   // the parent's latest update: level-0 values and state
        h->L[0].Avals = h->parent->L[0].Avals;
        h->updated = h->parent->updated;
    }
    if (!h->updated) return set_error(SG_ERR_STATE, "sg_amg_update must be called before sg_amg_apply");
    const cudaStream_t st = as_stream(stream);
    Level &L = h->L[0];
    const int64_t nd = L.n * L.b;
    int rc;
    const InstrToken tk = instr_begin(IK_AMG_APPLY, st);
    struct End {
        const InstrToken &t;
        cudaStream_t s;
        ~End() { instr_end(t, s); }
    } end{tk, st};
    if (h->opt.mixed) {
        k_to_float<<<grid_for(nd, 256), 256, 0, st>>>(nd, r, L.rhs32);
        rc = vcycle<float>(h, 0, st);
        if (!rc && h->corr_on) {
            rc = rect_spmv<float, float>(L.b, L.b, L.n, L.d_Arp, L.d_Acol, L.A32, L.x32, L.r32, 1.0, 0.0, L.rhs32, 1, st,
                                         L.Anblk);
            if (!rc) k_corr_apply<float><<<grid_for(L.n, 256), 256, 0, st>>>(L.n, h->corrC32, L.r32, L.x32);
        }
        if (!rc) k_to_double<<<grid_for(nd, 256), 256, 0, st>>>(nd, L.x32, z);
    } else {
        SG_CUDA(cudaMemcpyAsync(L.rhs, r, sizeof(double) * nd, cudaMemcpyDeviceToDevice, st));
        rc = vcycle<double>(h, 0, st);
        if (!rc && h->corr_on) {
            LevelView<double> v = view<double>(L);
            rc = rect_spmv<double, double>(L.b, L.b, L.n, L.d_Arp, L.d_Acol, v.A, L.x, L.r, 1.0, 0.0, L.rhs, 1, st,
                                           L.Anblk);
            if (!rc) k_corr_apply<double><<<grid_for(L.n, 256), 256, 0, st>>>(L.n, h->corrC, L.r, L.x);
        }
        if (!rc) SG_CUDA(cudaMemcpyAsync(z, L.x, sizeof(double) * nd, cudaMemcpyDeviceToDevice, st));
    }
    SG_CUDA(cudaGetLastError());
    return rc;
}

// Node-wise correction after every cycle (no counterpart in the reference): with C set,
// sg_amg_apply returns z + C (r - A z) for the cycle's z, C given as n_rows 3 x 3 row-major
// blocks (device, FP64, copied; converted to FP32 for a mixed-precision hierarchy).  C = NULL
// switches it off.
extern "C" int sg_amg_set_correction(sg_amg *h, const double *Cb, void *stream) {
    SG_CHECK_ARG(h, "null argument");
    SG_CHECK_ARG(!h->parent || !Cb, "the learned correction is not available on a clone");
    if (!Cb) {
        h->corr_on = 0;
        return SG_OK;
    }
    Level &L = h->L[0];
    SG_CHECK_ARG(L.b == 3, "the node-wise correction needs 3 x 3 node blocks");
    const cudaStream_t st = as_stream(stream);
    const int64_t nv = L.n * 9;
    if (!h->corrC) SG_CUDA(sg::device_alloc(&h->corrC, sizeof(double) * nv));
    SG_CUDA(cudaMemcpyAsync(h->corrC, Cb, sizeof(double) * nv, cudaMemcpyDeviceToDevice, st));
    if (h->opt.mixed) {
        if (!h->corrC32) SG_CUDA(sg::device_alloc(&h->corrC32, sizeof(float) * nv));
        k_to_float<<<grid_for(nv, 256), 256, 0, st>>>(nv, h->corrC, h->corrC32);
        SG_CUDA(cudaGetLastError());
    }
    h->corr_on = 1;
    return SG_OK;
}

// info: [levels, dense size, then per level: block size, block rows, blocks] in the first
// 2 + 3*10 entries; from entry 32 on, per level: blocks of its prolongator P (0 on the coarsest)
extern "C" int sg_amg_info(const sg_amg *h, int64_t *info, int32_t cap) {
    SG_CHECK_ARG(h && info && cap >= 2, "bad argument");
    info[0] = (int64_t)h->L.size();
    info[1] = h->nc_dense;
    int k = 2;
    for (const auto &L : h->L) {
        if (k + 3 > 32 || k + 3 > cap) break;
        info[k++] = L.b;
        info[k++] = L.n;
        info[k++] = L.Anblk;
    }
    for (size_t l = 0; l < h->L.size() && 32 + (int)l < cap; ++l) info[32 + l] = h->L[l].P.nblk;
    return SG_OK;
}

// Copy level l's matrix values (and, if not the coarsest, P values) to host buffers for checks.
extern "C" int sg_amg_export(const sg_amg *h, int32_t l, int32_t *A_rp, int32_t *A_col, double *A_vals,
                             int32_t *P_rp, int32_t *P_col, double *P_vals) {
    SG_CHECK_ARG(h && l >= 0 && l < (int)h->L.size(), "bad level");
    const Level &L = h->L[l];
    const double *A = L.Aext ? L.Avals : L.Aown_vals;
    if (A_rp) SG_CUDA(cudaMemcpy(A_rp, L.d_Arp, sizeof(int32_t) * (L.n + 1), cudaMemcpyDeviceToHost));
    if (A_col) SG_CUDA(cudaMemcpy(A_col, L.d_Acol, sizeof(int32_t) * L.Anblk, cudaMemcpyDeviceToHost));
    if (A_vals && A) SG_CUDA(cudaMemcpy(A_vals, A, sizeof(double) * L.Anblk * L.b * L.b, cudaMemcpyDeviceToHost));
    if (l + 1 < (int)h->L.size()) {
        if (P_rp) memcpy(P_rp, L.P.rp.data(), sizeof(int32_t) * (L.n + 1));
        if (P_col) memcpy(P_col, L.P.col.data(), sizeof(int32_t) * L.P.nblk);
        if (P_vals) SG_CUDA(cudaMemcpy(P_vals, L.Pv, sizeof(double) * L.P.nblk * L.b * L.bc, cudaMemcpyDeviceToHost));
    }
    return SG_OK;
}
