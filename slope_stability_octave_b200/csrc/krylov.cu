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
    // graph-replayed solve (dfgmres_graph): one CUDA graph holds the start, the iteration loop
    // (a conditional WHILE node whose body is one FGMRES iteration) and the small
    // least-squares solve; it is captured once per (matrix, preconditioner) and replayed
    double *u = nullptr;        // n: A z during its orthogonalisation
    int32_t *dstate = nullptr;  // [0] iterations done (j), [1] deflation columns k, [2] maxit
    double *dscal = nullptr;    // [0] |b|, [1] relative residual, [2] tol, [3] scale of the new basis vector,
                                // [4] b'b, [5] r0'r0
    double *dH = nullptr, *dcs = nullptr, *dsn = nullptr, *dg = nullptr, *dy = nullptr, *dhist = nullptr;
    const double **dptr = nullptr;  // [0] W, [1] A W of the current solve
    cudaStream_t cap = nullptr, cap2 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    uint64_t gkey = 0;
    int64_t launches_start = 0, launches_body = 0, launches_end = 0;
    int use_graph = 1;
    // blocked A-orthogonalisation: A times the block's input columns (n x 16), the block's
    // coefficients against earlier columns (256 x 16) and the per-CTA partial sums
    double *atb = nullptr, *cblk = nullptr, *tspart = nullptr;
    // Gram-matrix A-orthogonalisation (default, aorth_mode 1): G, T, the output-ordered T and
    // the output columns' processing indices (3 kcap^2 + kcap), the Gram partial sums
    // (GR_CTAS x 64 x 64) and the kept count on the device
    double *gram = nullptr, *gpart = nullptr;
    int32_t *gkout = nullptr;
    double *spy = nullptr;      // n x 16: interleaved products of the long-vector SpMM
    int aorth_mode = 1;
};

namespace sg {

static int ensure_kcap(sg_krylov *ws, int64_t k) {
    if (k <= ws->kcap) return SG_OK;
    const int64_t cap = std::max<int64_t>(k, std::max<int64_t>(64, ws->kcap * 2));
    double *part = nullptr, *hd = nullptr, *Wo = nullptr, *AWo = nullptr, *nt = nullptr, *sig = nullptr;
    const int64_t rows = std::max<int64_t>(cap, ws->maxit + 2);
    SG_CUDA(sg::device_alloc(&part, sizeof(double) * DOT_BLOCKS * rows));
    SG_CUDA(sg::device_alloc(&hd, sizeof(double) * (cap + 8)));
    SG_CUDA(sg::device_alloc(&Wo, sizeof(double) * ws->n * cap));
    SG_CUDA(sg::device_alloc(&AWo, sizeof(double) * ws->n * cap));
    SG_CUDA(sg::device_alloc(&nt, sizeof(double) * (cap + 8)));
    SG_CUDA(sg::device_alloc(&sig, sizeof(double) * (cap + 8)));
    double *gram = nullptr;
    SG_CUDA(sg::device_alloc(&gram, sizeof(double) * (3 * cap * cap + cap)));
    cudaFree(ws->gram);
    ws->gram = gram;
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

// ------------------------------------------------------------------ graph-replayed solve

// the basis column j (j read from the device) into w, and back
__global__ void k_col_get(int64_t n, const double *__restrict__ V, const int32_t *__restrict__ j,
                          double *__restrict__ w) {
    const double *c = V + (int64_t)j[0] * n;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        w[r] = c[r];
}
__global__ void k_col_put(int64_t n, const double *__restrict__ w, double *__restrict__ V,
                          const int32_t *__restrict__ j, const double *__restrict__ scale) {
    double *c = V + (int64_t)j[0] * n;
    const double s = scale ? scale[0] : 1.0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        c[r] = scale ? w[r] * s : w[r];
}

__global__ void k_fg_params(int32_t *st, double *sc, const double **ptrs, double tol, int maxit, int k,
                            const double *W, const double *AW) {
    st[0] = 0;
    st[1] = k;
    st[2] = maxit;
    sc[2] = tol;
    ptrs[0] = W;
    ptrs[1] = AW;
}

// start of the loop: |b|, |r0|, the first residual estimate, g = (|r0|, 0, ...), and whether
// to iterate at all (dfgmres_solver.m: no iteration when |r0| / |b| < tol)
__global__ void k_fg_start(cudaGraphConditionalHandle h, int mcap, int32_t *st, double *sc, double *g,
                           double *hist) {
    if (threadIdx.x != 0) return;
    double b_norm = sqrt(sc[4]);
    if (b_norm == 0.0) b_norm = 1.0;
    const double res = sqrt(sc[5]);
    const double rel = res / b_norm;
    sc[0] = b_norm;
    sc[1] = rel;
    hist[0] = rel;
    g[0] = res;
    for (int i = 1; i <= mcap; ++i) g[i] = 0.0;
    st[0] = 0;
    const bool go = (rel >= sc[2]) && st[2] > 0;
    sc[3] = go ? 1.0 / res : 0.0;
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

// End of iteration j: the new Hessenberg column (the two CGS passes' coefficients), the
// previous Givens rotations and a new one, the residual estimate |g_{j+1}| / |b|, the scale of
// the next basis vector and the loop condition -- the host loop's arithmetic, on the device.
__global__ void k_fg_arnoldi(cudaGraphConditionalHandle h, int mcap, int32_t *st, double *sc,
                             const double *__restrict__ h1, const double *__restrict__ h2,
                             const double *__restrict__ hn, double *H, double *cs, double *sn, double *g,
                             double *hist) {
    if (threadIdx.x != 0) return;
    const int j = st[0];
    for (int i = 0; i <= j; ++i) H[(size_t)i * mcap + j] = h1[i] + h2[i];
    const double hjj = sqrt(hn[0]);
    H[(size_t)(j + 1) * mcap + j] = hjj;
    for (int i = 0; i < j; ++i) {
        const double a = H[(size_t)i * mcap + j], bb = H[(size_t)(i + 1) * mcap + j];
        H[(size_t)i * mcap + j] = cs[i] * a + sn[i] * bb;
        H[(size_t)(i + 1) * mcap + j] = -sn[i] * a + cs[i] * bb;
    }
    const double a = H[(size_t)j * mcap + j], bb = H[(size_t)(j + 1) * mcap + j];
    const double den = hypot(a, bb);
    cs[j] = den > 0 ? a / den : 1.0;
    sn[j] = den > 0 ? bb / den : 0.0;
    H[(size_t)j * mcap + j] = den;
    H[(size_t)(j + 1) * mcap + j] = 0.0;
    g[j + 1] = -sn[j] * g[j];
    g[j] = cs[j] * g[j];
    const double rr = fabs(g[j + 1]) / sc[0];
    hist[j + 1] = rr;
    sc[1] = rr;
    const bool broke = hjj < 1e-14;   // happy breakdown (dfgmres_solver.m: H(j+1,j) < 1e-14)
    sc[3] = broke ? 0.0 : 1.0 / hjj;
    st[0] = j + 1;
    const bool go = !broke && !(rr < sc[2]) && (j + 1) < st[2];
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

// y = R \ g over the iterations done
__global__ void k_fg_solve_y(int mcap, const int32_t *st, const double *H, const double *g, double *y) {
    if (threadIdx.x != 0) return;
    const int it = st[0];
    for (int i = it - 1; i >= 0; --i) {
        double s = g[i];
        for (int c = i + 1; c < it; ++c) s -= H[(size_t)i * mcap + c] * y[c];
        y[i] = H[(size_t)i * mcap + i] != 0.0 ? s / H[(size_t)i * mcap + i] : 0.0;
    }
}

uint64_t amg_capture_key(const sg_amg *h);

static int graph_alloc(sg_krylov *ws) {
    if (ws->dstate) return SG_OK;
    const int m = ws->maxit;
    SG_CUDA(device_alloc(&ws->u, sizeof(double) * ws->n));
    SG_CUDA(device_alloc(&ws->dstate, sizeof(int32_t) * 8));
    SG_CUDA(device_alloc(&ws->dscal, sizeof(double) * 8));
    SG_CUDA(device_alloc(&ws->dH, sizeof(double) * (size_t)(m + 1) * m));
    SG_CUDA(device_alloc(&ws->dcs, sizeof(double) * m));
    SG_CUDA(device_alloc(&ws->dsn, sizeof(double) * m));
    SG_CUDA(device_alloc(&ws->dg, sizeof(double) * (m + 1)));
    SG_CUDA(device_alloc(&ws->dy, sizeof(double) * m));
    SG_CUDA(device_alloc(&ws->dhist, sizeof(double) * (m + 1)));
    SG_CUDA(device_alloc(&ws->dptr, sizeof(double *) * 2));
    SG_CUDA(cudaStreamCreateWithFlags(&ws->cap, cudaStreamNonBlocking));
    SG_CUDA(cudaStreamCreateWithFlags(&ws->cap2, cudaStreamNonBlocking));
    return SG_OK;
}

static void graph_release(sg_krylov *ws) {
    if (ws->gexec) cudaGraphExecDestroy(ws->gexec);
    if (ws->graph) cudaGraphDestroy(ws->graph);
    ws->gexec = nullptr;
    ws->graph = nullptr;
    ws->gkey = 0;
}

// Captures start, loop and least-squares solve for (A, Avals, M) into ws->gexec.
static int graph_capture(sg_krylov *ws, const sg_bsr *A, const double *Avals, sg_amg *M) {
    graph_release(ws);
    const int64_t n = ws->n;
    const int m = ws->maxit;
    const int kcap = (int)ws->kcap;
    double *h1 = ws->hdev, *h2 = ws->hdev + (m + 2), *hn = ws->hdev + 2 * (m + 2);
    InstrSuspend quiet;   // no event records inside the graph
    int rc = SG_OK;
    cudaStream_t cap = ws->cap, cap2 = ws->cap2;
    SG_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t g = nullptr;
    auto abort_capture = [&](int code) {
        cudaGraph_t dead = nullptr;
        cudaStreamEndCapture(cap, &dead);
        if (dead) cudaGraphDestroy(dead);
        cudaGetLastError();
        return code;
    };
    cudaStreamCaptureStatus status;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    if (cudaStreamGetCaptureInfo(cap, &status, nullptr, &g, &deps, &ndeps) != cudaSuccess)
        return abort_capture(set_error(SG_ERR_CUDA, "capture info"));
    cudaGraphConditionalHandle hcond;
    if (cudaGraphConditionalHandleCreate(&hcond, g, 0, cudaGraphCondAssignDefault) != cudaSuccess)
        return abort_capture(set_error(SG_ERR_CUDA, "conditional handle"));
    const int64_t l0 = sg_launch_count(0);
    count_launch(1);
    k_fg_start<<<1, 32, 0, cap>>>(hcond, m, ws->dstate, ws->dscal, ws->dg, ws->dhist);
    if (scale_dev(n, ws->V, ws->dscal + 3, 0, ws->V, cap) || cudaGetLastError() != cudaSuccess)
        return abort_capture(set_error(SG_ERR_CUDA, "capture start"));
    const int64_t l1 = sg_launch_count(0);
    if (cudaStreamGetCaptureInfo(cap, &status, nullptr, &g, &deps, &ndeps) != cudaSuccess)
        return abort_capture(set_error(SG_ERR_CUDA, "capture info"));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hcond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    if (cudaGraphAddNode(&cnode, g, deps, ndeps, &cp) != cudaSuccess)
        return abort_capture(set_error(SG_ERR_CUDA, "conditional node"));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if (cudaStreamUpdateCaptureDependencies(cap, &cnode, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
        return abort_capture(set_error(SG_ERR_CUDA, "capture dependencies"));
    // one iteration, captured into the loop body
    if (cudaStreamBeginCaptureToGraph(cap2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return abort_capture(set_error(SG_ERR_CUDA, "body capture"));
    {
        k_col_get<<<grid_for(n, 256, 8), 256, 0, cap2>>>(n, ws->V, ws->dstate, ws->w);
        if (M) rc = sg_amg_apply(M, ws->w, ws->t, cap2);
        else if (cudaMemcpyAsync(ws->t, ws->w, sizeof(double) * n, cudaMemcpyDeviceToDevice, cap2) != cudaSuccess)
            rc = set_error(SG_ERR_CUDA, "body copy");
        if (!rc) rc = multidot_dc(n, ws->dstate + 1, 0, kcap, nullptr, ws->dptr + 1, n, ws->t, ws->part, ws->hd, cap2);
        if (!rc) rc = gemv_dc(-1, n, ws->dstate + 1, 0, kcap, nullptr, ws->dptr, n, ws->hd, ws->t, cap2);
        if (!rc) k_col_put<<<grid_for(n, 256, 8), 256, 0, cap2>>>(n, ws->t, ws->Z, ws->dstate, nullptr);
        if (!rc) rc = bsr_spmv<double, double>(*A, Avals, ws->t, ws->u, 1.0, 0.0, cap2);
        if (!rc) rc = multidot_dc(n, ws->dstate, 1, m, ws->V, nullptr, n, ws->u, ws->part, h1, cap2);
        if (!rc) rc = gemv_dc(-1, n, ws->dstate, 1, m, ws->V, nullptr, n, h1, ws->u, cap2);
        if (!rc) rc = multidot_dc(n, ws->dstate, 1, m, ws->V, nullptr, n, ws->u, ws->part, h2, cap2);
        if (!rc) rc = gemv_dc(-1, n, ws->dstate, 1, m, ws->V, nullptr, n, h2, ws->u, cap2);
        if (!rc) rc = multidot(n, 1, ws->u, n, ws->u, ws->part, hn, cap2);
        if (!rc) {
            count_launch(1);
            k_fg_arnoldi<<<1, 32, 0, cap2>>>(hcond, m, ws->dstate, ws->dscal, h1, h2, hn, ws->dH, ws->dcs, ws->dsn,
                                             ws->dg, ws->dhist);
            k_col_put<<<grid_for(n, 256, 8), 256, 0, cap2>>>(n, ws->u, ws->V, ws->dstate, ws->dscal + 3);
        }
        cudaGraph_t body_out = nullptr;
        const cudaError_t e = cudaStreamEndCapture(cap2, &body_out);
        if (!rc && (e != cudaSuccess || cudaGetLastError() != cudaSuccess)) rc = set_error(SG_ERR_CUDA, "body capture");
    }
    if (rc) return abort_capture(rc);
    const int64_t l2 = sg_launch_count(0);
    count_launch(1);
    k_fg_solve_y<<<1, 32, 0, cap>>>(m, ws->dstate, ws->dH, ws->dg, ws->dy);
    cudaGraph_t full = nullptr;
    if (cudaStreamEndCapture(cap, &full) != cudaSuccess || !full) {
        if (full) cudaGraphDestroy(full);
        cudaGetLastError();
        return set_error(SG_ERR_CUDA, "graph capture");
    }
    cudaGraphExec_t ex = nullptr;
    if (cudaGraphInstantiate(&ex, full, 0) != cudaSuccess) {
        cudaGraphDestroy(full);
        cudaGetLastError();
        return set_error(SG_ERR_CUDA, "graph instantiation");
    }
    const int64_t l3 = sg_launch_count(0);
    ws->graph = full;
    ws->gexec = ex;
    ws->launches_start = l1 - l0;
    ws->launches_body = l2 - l1;
    ws->launches_end = l3 - l2;
    // the captured launches were counted at capture; executions are counted per solve instead
    count_launch((int)-(l3 - l0));
    return SG_OK;
}

static uint64_t graph_key(const sg_krylov *ws, const sg_bsr *A, const double *Avals, sg_amg *M) {
    uint64_t k = (uint64_t)(uintptr_t)A * 1000003u ^ (uint64_t)(uintptr_t)Avals * 10007u;
    k ^= (uint64_t)(uintptr_t)ws->part * 131u ^ (uint64_t)(uintptr_t)ws->hd * 137u ^ (uint64_t)ws->kcap * 7919u;
    if (M) k ^= amg_capture_key(M) * 1315423911u;
    return k | 1u;
}

// The graph-replayed solve: the same start, iterations, stopping test and least-squares
// solution as the host loop of sg_dfgmres_solve, with one host synchronisation per solve
// instead of one per iteration.
static int dfgmres_graph(sg_krylov *ws, const sg_bsr *A, const double *Avals, sg_amg *M, const double *Wd,
                         const double *AWd, int32_t k, const double *b, double *x, double tol, int32_t maxit,
                         int32_t *iters, double *relres, double *res_hist, cudaStream_t st) {
    const int64_t n = ws->n;
    int rc = graph_alloc(ws);
    if (rc) return rc;
    const uint64_t key = graph_key(ws, A, Avals, M);
    if (!ws->gexec || ws->gkey != key) {
        rc = graph_capture(ws, A, Avals, M);
        if (rc) return rc;
        ws->gkey = key;
    }
    // x0 = Wd (Wd' b), r0 = b - A x0 = V(:, 0), b'b and r0'r0, the solve's parameters
    SG_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
    if (k > 0) {
        if ((rc = multidot(n, k, Wd, n, b, ws->part, ws->hd, st))) return rc;
        if ((rc = gemv_add(n, k, Wd, n, ws->hd, x, st))) return rc;
    }
    if ((rc = bsr_residual<double, double>(*A, Avals, x, b, ws->V, st))) return rc;
    if ((rc = multidot(n, 1, b, n, b, ws->part, ws->dscal + 4, st))) return rc;
    if ((rc = multidot(n, 1, ws->V, n, ws->V, ws->part, ws->dscal + 5, st))) return rc;
    count_launch(1);
    k_fg_params<<<1, 1, 0, st>>>(ws->dstate, ws->dscal, ws->dptr, tol, maxit, k, Wd, AWd);
    SG_CUDA(cudaGetLastError());
    SG_CUDA(cudaGraphLaunch(ws->gexec, st));
    if ((rc = gemv_dc(1, n, ws->dstate, 0, ws->maxit, ws->Z, nullptr, n, ws->dy, x, st))) return rc;
    double *hp = ws->hpin;
    int32_t *ip = reinterpret_cast<int32_t *>(hp + ws->maxit + 4);
    SG_CUDA(cudaMemcpyAsync(ip, ws->dstate, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaMemcpyAsync(hp, ws->dscal + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (res_hist) SG_CUDA(cudaMemcpyAsync(hp + 1, ws->dhist, sizeof(double) * (maxit + 1), cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    const int it = ip[0];
    count_launch((int)(ws->launches_start + ws->launches_body * it + ws->launches_end));
    *iters = it;
    if (relres) *relres = hp[0];
    if (res_hist)
        for (int i = 0; i <= it; ++i) res_hist[i] = hp[1 + i];
    return SG_OK;
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
    graph_release(ws);
    cudaFree(ws->atb); cudaFree(ws->cblk); cudaFree(ws->tspart);
    cudaFree(ws->gram); cudaFree(ws->gpart); cudaFree(ws->gkout); cudaFree(ws->spy);
    cudaFree(ws->u); cudaFree(ws->dstate); cudaFree(ws->dscal); cudaFree(ws->dH); cudaFree(ws->dcs);
    cudaFree(ws->dsn); cudaFree(ws->dg); cudaFree(ws->dy); cudaFree(ws->dhist); cudaFree(ws->dptr);
    if (ws->cap) cudaStreamDestroy(ws->cap);
    if (ws->cap2) cudaStreamDestroy(ws->cap2);
    if (ws->hpin) cudaFreeHost(ws->hpin);
    cudaSetDevice(cur);
    delete ws;
    return SG_OK;
}

// 1: solves run as a replayed CUDA graph (default); 0: the host-driven loop, one host
// synchronisation per iteration (same arithmetic)
extern "C" int sg_krylov_set_graph(sg_krylov *ws, int32_t on) {
    SG_CHECK_ARG(ws, "null workspace");
    ws->use_graph = on != 0;
    return SG_OK;
}

// 1: the A-orthogonalisation through the Gram matrix (default); 0: the column-blocked
// Gram-Schmidt (coefficients and norms from n-long vector passes per column)
extern "C" int sg_krylov_set_aorth(sg_krylov *ws, int32_t mode) {
    SG_CHECK_ARG(ws && (mode == 0 || mode == 1), "bad argument");
    ws->aorth_mode = mode;
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
    if (ws->use_graph && (k == 0 || AWd))
        return dfgmres_graph(ws, A, Avals, M, Wd, AWd, k, b, x, tol, maxit, iters, relres, res_hist, st);
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
    const InstrToken tk_all = instr_begin(IK_AORTH, st);
    instr_units(IK_AORTH, k);
    struct EndAll {
        const InstrToken &t;
        cudaStream_t s;
        ~EndAll() { instr_end(t, s); }
    } end_all{tk_all, st};
    int rc = ensure_kcap(ws, k);
    if (rc) return rc;
    // Wo, AWo: the A-orthonormalised columns and A times them, in processing order; nt[i] is
    // column i's A-norm^2 and sig[i] its sign (kept, scaled and signed on the device, so the
    // loop needs no host round trip; dropped columns are left as zeros).
    double *Wo = ws->Worth, *AWo = ws->AWorth, *part = ws->part, *c = ws->hd;
    double *nt = ws->nt, *sig = ws->sig;
    const unsigned gb = grid_for(n, 256, 8);
    // A times every input column up front (processing order i takes column k - 1 - i): the
    // products do not depend on the orthogonalisation, and one SpMM reads A once per eight
    // columns where a SpMV per column reads it k times
    if (A->b == 3 && k >= 4 && (double)n * 8 * 8 > 48e6) {
        // long vectors: interleaved copies of 16 columns (scratch: the block buffer and spy)
        if (!ws->atb) {
            SG_CUDA(device_alloc(&ws->atb, sizeof(double) * n * 16));
            SG_CUDA(device_alloc(&ws->cblk, sizeof(double) * 256 * 16));
            SG_CUDA(device_alloc(&ws->tspart, sizeof(double) * TS_PART_CTAS * 256 * 16));
        }
        if (!ws->spy) SG_CUDA(device_alloc(&ws->spy, sizeof(double) * n * 16));
        rc = bsr_spmm_interleaved(*A, Avals, W + (int64_t)(k - 1) * n, -n, AWo, n, k, ws->atb, ws->spy, st);
    } else if (A->b == 3) {
        rc = bsr_spmm(*A, Avals, W + (int64_t)(k - 1) * n, -n, AWo, n, k, st);
    } else {
        for (int i = 0; i < k && !rc; ++i)
            rc = bsr_spmv<double, double>(*A, Avals, W + (int64_t)(k - 1 - i) * n, AWo + (int64_t)i * n, 1.0, 0.0, st);
    }
    if (rc) return rc;
    if (ws->aorth_mode == 1) {
        // Gram matrix, recurrence on one CTA, then U = S T into Wo and A U = (A S) T into AW
        if (!ws->gpart) {
            SG_CUDA(device_alloc(&ws->gpart, sizeof(double) * GR_CTAS * 64 * 64));
            SG_CUDA(device_alloc(&ws->gkout, sizeof(int32_t) * 4));
        }
        double *G = ws->gram, *Tp = G + (int64_t)k * k, *Ta = Tp + (int64_t)k * k;
        int32_t *pmap = reinterpret_cast<int32_t *>(Ta + (int64_t)k * k);
        const double *S = W + (int64_t)(k - 1) * n;   // processing order: column i is W's k - 1 - i
        if ((rc = gram_upper(n, k, S, -n, AWo, n, G, ws->gpart, st))) return rc;
        if ((rc = gram_recurrence(k, G, Tp, eps_add, Ta, nt, sig, ws->gkout, pmap, st))) return rc;
        if ((rc = ts_apply(n, k, ws->gkout, pmap, S, -n, Ta, Wo, n, st))) return rc;
        if (AW && (rc = ts_apply(n, k, ws->gkout, pmap, AWo, n, Ta, AW, n, st))) return rc;
        int32_t ko = 0;
        SG_CUDA(cudaMemcpyAsync(&ko, ws->gkout, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        SG_CUDA(cudaStreamSynchronize(st));
        if (ko > 0)
            SG_CUDA(cudaMemcpyAsync(W, Wo, sizeof(double) * n * ko, cudaMemcpyDeviceToDevice, st));
        *k_out = ko;
        SG_CUDA(cudaStreamSynchronize(st));
        return SG_OK;
    }
    // Blocked one-pass Gram-Schmidt (aorth_mode 0): columns are processed in blocks of AORTH_BLOCK; a block's
    // coefficients against all earlier (final) columns come from one tall-skinny product
    // c = diag(sig) U' (A S_blk), applied to the block's columns and their A-images by two more,
    // then the columns inside the block are treated one after another as before.  Every
    // coefficient is sig_j (A src_i)' u_j as in the column-by-column loop, so the result is the
    // same one-pass A-orthogonalisation summed in another order; the earlier columns are read
    // a few times per block instead of three times per column.
    constexpr int AORTH_BLOCK = 16;
    if (!ws->atb) {
        SG_CUDA(device_alloc(&ws->atb, sizeof(double) * n * AORTH_BLOCK));
        SG_CUDA(device_alloc(&ws->cblk, sizeof(double) * 256 * AORTH_BLOCK));
        SG_CUDA(device_alloc(&ws->tspart, sizeof(double) * TS_PART_CTAS * 256 * AORTH_BLOCK));
    }
    for (int i0 = 0; i0 < k && !rc; i0 += AORTH_BLOCK) {
        const int b = std::min(AORTH_BLOCK, k - i0);
        double *WoB = Wo + (int64_t)i0 * n, *AWoB = AWo + (int64_t)i0 * n;
        // A src of the block's columns (kept: AWo's columns change below) and src itself
        SG_CUDA(cudaMemcpyAsync(ws->atb, AWoB, sizeof(double) * n * b, cudaMemcpyDeviceToDevice, st));
        for (int l = 0; l < b; ++l)
            SG_CUDA(cudaMemcpyAsync(WoB + (int64_t)l * n, W + (int64_t)(k - 1 - i0 - l) * n, sizeof(double) * n,
                                    cudaMemcpyDeviceToDevice, st));
        for (int j0 = 0; j0 < i0 && !rc; j0 += 256) {
            const int mj = std::min(256, i0 - j0);
            rc = gemm_tn(n, mj, b, Wo + (int64_t)j0 * n, n, ws->atb, n, sig + j0, ws->cblk, mj, ws->tspart, st);
            if (!rc) rc = gemm_nn_sub(n, mj, b, Wo + (int64_t)j0 * n, n, ws->cblk, mj, WoB, n, st);
            if (!rc) rc = gemm_nn_sub(n, mj, b, AWo + (int64_t)j0 * n, n, ws->cblk, mj, AWoB, n, st);
        }
        for (int l = 0; l < b && !rc; ++l) {
            const int i = i0 + l;
            const double *At_i = ws->atb + (int64_t)l * n;
            double *col_i = Wo + (int64_t)i * n, *acol_i = AWo + (int64_t)i * n;
            if (l > 0) {
                // c_j = sig_j (A src)' u_j for the block's earlier columns
                if ((rc = multidot(n, l, WoB, n, At_i, part, c, st))) break;
                count_launch();
                k_mul_sign<<<1, 256, 0, st>>>(l, c, sig + i0);
                if ((rc = gemv_sub(n, l, WoB, n, c, col_i, st))) break;
                if ((rc = gemv_sub(n, l, AWoB, n, c, acol_i, st))) break;
            }
            if ((rc = multidot(n, 1, col_i, n, At_i, part, nt + i, st))) break;
            k_anorm_scale<<<gb, 256, 0, st>>>(n, nt + i, eps_add, col_i, col_i, acol_i, sig + i);
            SG_CUDA(cudaGetLastError());
        }
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
