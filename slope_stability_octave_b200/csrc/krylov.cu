// (c1, c3) Deflated flexible GMRES and A-orthogonalisation of the deflation basis.
//
//   sg_dfgmres_solve     +LINEAR_SOLVERS/dfgmres_solver.m:1-181
//       x0 = W (W' b) and Proj(w) = w - W (W' (A w)) when a deflation basis W is given;
//       no restart, maxit iterations; flexible: the preconditioned vectors z_j are stored
//       and x = x0 + Z y.  Orthogonalisation is classical Gram-Schmidt applied twice (CGS2:
//       two passes of one multi-dot and one GEMV each) instead of the reference's modified
//       Gram-Schmidt loop -- the same projection with MGS-level stability in 4 sweeps
//       over the basis instead of 2(j+1).  The small least-squares problem is solved with
//       Givens rotations on the host (the reference re-solves H \ g each step; same y).
//   sg_a_orthogonalize   +LINEAR_SOLVERS/A_orthogonalize.m:1-58 (columns processed last
//       to first, one-pass A-orthogonalisation against the kept columns, columns with
//       |w'Aw| <= eps dropped, output reversed)
//
// Vectors and bases are device arrays; bases are column-major with leading dimension n.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "instr.cuh"
#include "linalg.cuh"
#include "mesh.h"
#include "sg_common.cuh"

struct sg_amg;
extern "C" int sg_amg_apply(sg_amg *h, const double *r, double *z, void *stream);

struct sg_krylov {
    int64_t n = 0;
    int32_t maxit = 0;
    double *V = nullptr, *Z = nullptr, *w = nullptr, *t = nullptr;
    double *part = nullptr;     // DOT_BLOCKS * max(maxit + 2, kcap)
    double *hdev = nullptr;     // 2 * (maxit + 2) + 4 scalars
    double *hd = nullptr;       // kcap coefficients for the deflation projection
    double *Worth = nullptr;    // n * kcap
    double *AWorth = nullptr;   // n * kcap
    double *nt = nullptr, *sig = nullptr;  // kcap A-norms^2 and signs
    int64_t kcap = 0;
    double *hpin = nullptr;     // pinned host mirror of hdev
    int device = 0;
};

namespace sg {

static int ensure_kcap(sg_krylov *ws, int64_t k) {
    if (k <= ws->kcap) return SG_OK;
    const int64_t cap = std::max<int64_t>(k, ws->kcap * 2 + 16);
    double *part = nullptr, *hd = nullptr, *Wo = nullptr, *AWo = nullptr, *nt = nullptr, *sig = nullptr;
    const int64_t rows = std::max<int64_t>(cap, ws->maxit + 2);
    SG_CUDA(sg::device_alloc(&part, sizeof(double) * DOT_BLOCKS * rows));
    SG_CUDA(sg::device_alloc(&hd, sizeof(double) * (cap + 8)));
    SG_CUDA(sg::device_alloc(&Wo, sizeof(double) * ws->n * cap));
    SG_CUDA(sg::device_alloc(&AWo, sizeof(double) * ws->n * cap));
    SG_CUDA(sg::device_alloc(&nt, sizeof(double) * (cap + 8)));
    SG_CUDA(sg::device_alloc(&sig, sizeof(double) * (cap + 8)));
    cudaFree(ws->part);
    cudaFree(ws->hd);
    cudaFree(ws->Worth);
    cudaFree(ws->AWorth);
    cudaFree(ws->nt);
    cudaFree(ws->sig);
    ws->part = part;
    ws->hd = hd;
    ws->Worth = Wo;
    ws->AWorth = AWo;
    ws->nt = nt;
    ws->sig = sig;
    ws->kcap = cap;
    return SG_OK;
}

__global__ void k_scale_host(int64_t n, double s, const double *__restrict__ x, double *__restrict__ y) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        y[r] = x[r] * s;
}

// c[j] *= norms[j] (norms = +-1 signature of the A-orthogonal basis)
__global__ void k_mul_sign(int m, double *__restrict__ c, const double *__restrict__ sign) {
    for (int j = threadIdx.x; j < m; j += blockDim.x) c[j] *= sign[j];
}

// Keep a column when |nt| > eps: u = tmp / sqrt|nt|, A u = atmp / sqrt|nt|, sign = sign(nt);
// otherwise u = A u = 0 (A_orthogonalize.m:40-52).
__global__ void k_anorm_scale(int64_t n, const double *__restrict__ ntp, double eps, const double *__restrict__ tmp,
                              double *__restrict__ col, double *__restrict__ acol, double *__restrict__ sgn) {
    const double nt = ntp[0];
    const bool keep = fabs(nt) > eps;
    const double s = keep ? 1.0 / sqrt(fabs(nt)) : 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) sgn[0] = (keep && nt < 0.0) ? -1.0 : 1.0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        col[r] = tmp[r] * s;
        acol[r] = acol[r] * s;
    }
}

}  // namespace sg

using namespace sg;

extern "C" int sg_krylov_create(int64_t n, int32_t maxit, sg_krylov **out) {
    SG_CHECK_ARG(out && n > 0 && maxit > 0 && maxit <= 2000, "bad Krylov workspace size");
    *out = nullptr;
    sg_krylov *ws = new (std::nothrow) sg_krylov();
    if (!ws) return set_error(SG_ERR_NOMEM, "host allocation");
    ws->n = n;
    ws->maxit = maxit;
    cudaGetDevice(&ws->device);
    cudaError_t e = sg::device_alloc(&ws->V, sizeof(double) * n * (maxit + 1));
    if (!e) e = sg::device_alloc(&ws->Z, sizeof(double) * n * maxit);
    if (!e) e = sg::device_alloc(&ws->w, sizeof(double) * n);
    if (!e) e = sg::device_alloc(&ws->t, sizeof(double) * n);
    if (!e) e = sg::device_alloc(&ws->hdev, sizeof(double) * (2 * (maxit + 2) + 8));
    if (!e) e = cudaMallocHost(&ws->hpin, sizeof(double) * (2 * (maxit + 2) + 8));
    int rc = e ? cuda_error(e, "Krylov workspace") : ensure_kcap(ws, 16);
    if (rc) {
        cudaFree(ws->V); cudaFree(ws->Z); cudaFree(ws->w); cudaFree(ws->t); cudaFree(ws->hdev);
        if (ws->hpin) cudaFreeHost(ws->hpin);
        delete ws;
        return rc;
    }
    *out = ws;
    return SG_OK;
}

extern "C" int sg_krylov_destroy(sg_krylov *ws) {
    if (!ws) return SG_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(ws->device);
    cudaFree(ws->V); cudaFree(ws->Z); cudaFree(ws->w); cudaFree(ws->t); cudaFree(ws->hdev);
    cudaFree(ws->part); cudaFree(ws->hd); cudaFree(ws->Worth); cudaFree(ws->AWorth); cudaFree(ws->nt);
    cudaFree(ws->sig);
    if (ws->hpin) cudaFreeHost(ws->hpin);
    cudaSetDevice(cur);
    delete ws;
    return SG_OK;
}

// Solve A x = b.  M: AMG preconditioner or NULL (identity).  Wd: n x k deflation basis
// (A-orthonormal, may be NULL with k = 0); AWd: A Wd or NULL (then one extra SpMV per
// iteration forms A z for the projection).  x is overwritten.  res_hist (optional, host,
// maxit + 1 entries) receives the relative residual estimates.
extern "C" int sg_dfgmres_solve(sg_krylov *ws, const sg_bsr *A, const double *Avals, sg_amg *M, const double *Wd,
                                const double *AWd, int32_t k, const double *b, double *x, double tol, int32_t maxit,
                                int32_t *iters, double *relres, double *res_hist, void *stream) {
    SG_CHECK_ARG(ws && A && Avals && b && x, "null argument");
    SG_CHECK_ARG(maxit > 0 && maxit <= ws->maxit, "maxit exceeds the workspace");
    SG_CHECK_ARG(k >= 0 && (k == 0 || Wd), "bad deflation basis");
    const int64_t n = ws->n;
    SG_CHECK_ARG(n == A->n_rows * A->b, "vector length does not match the matrix");
    const cudaStream_t st = as_stream(stream);
    int rc = ensure_kcap(ws, std::max<int64_t>(k, 1));
    if (rc) return rc;
    double *part = ws->part, *hdev = ws->hdev, *hp = ws->hpin;
    const unsigned gb = grid_for(n, 256, 8);
    // x0 = Wd (Wd' b) ; r0 = b - A x0
    SG_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
    if (k > 0) {
        if ((rc = multidot(n, k, Wd, n, b, part, ws->hd, st))) return rc;
        if ((rc = gemv_add(n, k, Wd, n, ws->hd, x, st))) return rc;
    }
    double *v0 = ws->V;
    if ((rc = bsr_residual<double, double>(*A, Avals, x, b, v0, st))) return rc;
    if ((rc = multidot(n, 1, b, n, b, part, hdev, st))) return rc;
    if ((rc = multidot(n, 1, v0, n, v0, part, hdev + 1, st))) return rc;
    SG_CUDA(cudaMemcpyAsync(hp, hdev, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    double b_norm = std::sqrt(hp[0]);
    if (b_norm == 0.0) b_norm = 1.0;
    double res = std::sqrt(hp[1]);
    if (res_hist) res_hist[0] = res / b_norm;
    if (!(res / b_norm >= tol)) {  // converged (or NaN: reported through relres)
        *iters = 0;
        if (relres) *relres = res / b_norm;
        return SG_OK;
    }
    k_scale_host<<<gb, 256, 0, st>>>(n, 1.0 / res, v0, v0);
    const int m = maxit;
    std::vector<double> H((size_t)(m + 1) * m, 0.0), cs(m), sn(m), g(m + 1, 0.0), y(m);
    g[0] = res;
    int it = 0;
    bool broke = false;
    for (int j = 0; j < m; ++j) {
        double *vj = ws->V + (int64_t)j * n, *zj = ws->Z + (int64_t)j * n, *u = ws->V + (int64_t)(j + 1) * n;
        // z = M v_j
        if (M) {
            if ((rc = sg_amg_apply(M, vj, zj, stream))) return rc;
        } else {
            SG_CUDA(cudaMemcpyAsync(zj, vj, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        }
        // z = z - Wd (Wd' (A z)); with AWd = A Wd given, Wd' (A z) = AWd' z (A symmetric)
        if (k > 0) {
            if (AWd) {
                if ((rc = multidot(n, k, AWd, n, zj, part, ws->hd, st))) return rc;
            } else {
                if ((rc = bsr_spmv<double, double>(*A, Avals, zj, ws->t, 1.0, 0.0, st))) return rc;
                if ((rc = multidot(n, k, Wd, n, ws->t, part, ws->hd, st))) return rc;
            }
            if ((rc = gemv_sub(n, k, Wd, n, ws->hd, zj, st))) return rc;
        }
        // u = A z ; CGS2 against v_0..v_j
        if ((rc = bsr_spmv<double, double>(*A, Avals, zj, u, 1.0, 0.0, st))) return rc;
        const int nv = j + 1;
        double *h1 = hdev, *h2 = hdev + (m + 2), *hn = hdev + 2 * (m + 2);
        if ((rc = multidot(n, nv, ws->V, n, u, part, h1, st))) return rc;
        if ((rc = gemv_sub(n, nv, ws->V, n, h1, u, st))) return rc;
        if ((rc = multidot(n, nv, ws->V, n, u, part, h2, st))) return rc;
        if ((rc = gemv_sub(n, nv, ws->V, n, h2, u, st))) return rc;
        if ((rc = multidot(n, 1, u, n, u, part, hn, st))) return rc;
        SG_CUDA(cudaMemcpyAsync(hp, hdev, sizeof(double) * (2 * (m + 2) + 1), cudaMemcpyDeviceToHost, st));
        SG_CUDA(cudaStreamSynchronize(st));
        for (int i = 0; i < nv; ++i) H[(size_t)i * m + j] = hp[i] + hp[(m + 2) + i];
        const double hjj = std::sqrt(hp[2 * (m + 2)]);
        H[(size_t)(j + 1) * m + j] = hjj;
        it = j + 1;
        // Givens: apply previous rotations, then a new one
        for (int i = 0; i < j; ++i) {
            const double a = H[(size_t)i * m + j], bb = H[(size_t)(i + 1) * m + j];
            H[(size_t)i * m + j] = cs[i] * a + sn[i] * bb;
            H[(size_t)(i + 1) * m + j] = -sn[i] * a + cs[i] * bb;
        }
        const double a = H[(size_t)j * m + j], bb = H[(size_t)(j + 1) * m + j];
        const double den = std::hypot(a, bb);
        cs[j] = den > 0 ? a / den : 1.0;
        sn[j] = den > 0 ? bb / den : 0.0;
        H[(size_t)j * m + j] = den;
        H[(size_t)(j + 1) * m + j] = 0.0;
        g[j + 1] = -sn[j] * g[j];
        g[j] = cs[j] * g[j];
        const double rr = std::fabs(g[j + 1]) / b_norm;
        if (res_hist) res_hist[j + 1] = rr;
        if (hjj < 1e-14) {  // happy breakdown (dfgmres_solver.m: H(j+1,j) < 1e-14)
            broke = true;
            res = rr;
            break;
        }
        k_scale_host<<<gb, 256, 0, st>>>(n, 1.0 / hjj, u, u);
        res = rr;
        if (rr < tol) break;
    }
    (void)broke;
    // y = R \ g (upper triangular, it x it)
    for (int i = it - 1; i >= 0; --i) {
        double s = g[i];
        for (int c = i + 1; c < it; ++c) s -= H[(size_t)i * m + c] * y[c];
        y[i] = H[(size_t)i * m + i] != 0.0 ? s / H[(size_t)i * m + i] : 0.0;
    }
    for (int i = 0; i < it; ++i) hp[i] = y[i];
    SG_CUDA(cudaMemcpyAsync(hdev, hp, sizeof(double) * it, cudaMemcpyHostToDevice, st));
    if ((rc = gemv_add(n, it, ws->Z, n, hdev, x, st))) return rc;
    SG_CUDA(cudaStreamSynchronize(st));
    *iters = it;
    if (relres) *relres = res;
    return SG_OK;
}

// A-orthonormalise the n x k basis W in place (column-major, ld = n); returns the number of
// kept columns in *k_out (W's first *k_out columns hold the result).  AW (optional, n x k)
// receives A times the kept columns, in the same order, for the solve's projection.
extern "C" int sg_a_orthogonalize(sg_krylov *ws, const sg_bsr *A, const double *Avals, double *W, double *AW,
                                  int32_t k, double eps_add, int32_t *k_out, void *stream) {
    SG_CHECK_ARG(ws && A && Avals && k_out && k >= 0 && (k == 0 || W), "bad argument");
    const int64_t n = ws->n;
    const cudaStream_t st = as_stream(stream);
    if (k == 0) { *k_out = 0; return SG_OK; }
    const InstrRedirect redirect(IK_SPMV3_F64, IK_SPMV3_F64_AORTH);
    int rc = ensure_kcap(ws, k);
    if (rc) return rc;
    // Wo, AWo: the A-orthonormalised columns and A times them, in processing order; nt[i] is
    // column i's A-norm^2 and sig[i] its sign (kept, scaled and signed on the device, so the
    // loop needs no host round trip; dropped columns are left as zeros).
    double *Wo = ws->Worth, *AWo = ws->AWorth, *At = ws->t, *tmp = ws->w, *part = ws->part, *c = ws->hd;
    double *nt = ws->nt, *sig = ws->sig;
    const unsigned gb = grid_for(n, 256, 8);
    // A times every input column up front (processing order i takes column k - 1 - i): the
    // products do not depend on the orthogonalisation, and one SpMM reads A once per eight
    // columns where a SpMV per column reads it k times
    if (A->b == 3) {
        rc = bsr_spmm(*A, Avals, W + (int64_t)(k - 1) * n, -n, AWo, n, k, st);
    } else {
        for (int i = 0; i < k && !rc; ++i)
            rc = bsr_spmv<double, double>(*A, Avals, W + (int64_t)(k - 1 - i) * n, AWo + (int64_t)i * n, 1.0, 0.0, st);
    }
    if (rc) return rc;
    for (int i = 0; i < k && !rc; ++i) {
        const double *src = W + (int64_t)(k - 1 - i) * n;
        double *col_i = Wo + (int64_t)i * n, *acol_i = AWo + (int64_t)i * n;
        SG_CUDA(cudaMemcpyAsync(At, acol_i, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        SG_CUDA(cudaMemcpyAsync(tmp, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        if (i > 0) {
            // c_j = sig_j (A src)' u_j ;  tmp -= sum c_j u_j ;  A tmp = A src - sum c_j A u_j
            if ((rc = multidot(n, i, Wo, n, At, part, c, st))) break;
            count_launch();
            k_mul_sign<<<1, 256, 0, st>>>(i, c, sig);
            if ((rc = gemv_sub(n, i, Wo, n, c, tmp, st))) break;
            if ((rc = gemv_sub(n, i, AWo, n, c, acol_i, st))) break;
        }
        if ((rc = multidot(n, 1, tmp, n, At, part, nt + i, st))) break;
        k_anorm_scale<<<gb, 256, 0, st>>>(n, nt + i, eps_add, tmp, col_i, acol_i, sig + i);
        SG_CUDA(cudaGetLastError());
    }
    if (rc) return rc;
    std::vector<double> nth(k);
    SG_CUDA(cudaMemcpyAsync(nth.data(), nt, sizeof(double) * k, cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    // kept columns, reversed: output column o = kept column in reverse processing order
    int o = 0;
    for (int i = k - 1; i >= 0; --i) {
        if (!(std::fabs(nth[i]) > eps_add)) continue;
        SG_CUDA(cudaMemcpyAsync(W + (int64_t)o * n, Wo + (int64_t)i * n, sizeof(double) * n,
                                cudaMemcpyDeviceToDevice, st));
        if (AW)
            SG_CUDA(cudaMemcpyAsync(AW + (int64_t)o * n, AWo + (int64_t)i * n, sizeof(double) * n,
                                    cudaMemcpyDeviceToDevice, st));
        ++o;
    }
    *k_out = o;
    SG_CUDA(cudaStreamSynchronize(st));
    return SG_OK;
}
