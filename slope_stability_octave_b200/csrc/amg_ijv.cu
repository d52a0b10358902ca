// (d1, d2) Preconditioner instances keyed by id over host COO triplets: the command set of
// the reference's hypre_boomeramg_mex (+LINEAR_SOLVERS/mex/hypre_boomeramg_mex.cpp):
//
//   sg_amg_setup_ijv      'setup_ijv', I, J, V, n, Z, opts, id   (:1013-1146)
//   sg_amg_update_values  'update_values', V, id                 (:1151-1213)
//   sg_amg_apply_host     'apply', r, id                         (:751-796)
//   sg_amg_clear          'clear' [, id]                         (:798-829)
//   sg_amg_ijv_info       'info'                                 (:830-853)
//
// Semantics kept from the reference: I and J are 1-based indices stored as doubles (Octave's
// numeric arrays), the triplets give the full (both-triangle) matrix, an id names a
// persistent instance, a repeated setup_ijv on an existing id with the same number of
// triplets reuses the pattern and only replaces the values (unless force_rebuild), a value
// update re-runs the numeric set-up, apply takes and returns host vectors of length n.
// Unknown ids and bad sizes return status codes (the reference raises hypre:* errors).
//
// Instead of BoomerAMG, an instance holds this library's smoothed-aggregation AMG over a
// node-block embedding of the matrix: the free DOFs are grouped into nodes by their
// component index (opts dof_func, as set_linear_solver.m builds it: mod(q - 1, 3) over the
// node-major free-DOF order; a DOF starts a new node when its component is not larger than
// the previous DOF's), and the matrix becomes a block matrix over those nodes with b x b
// blocks (b = num_functions) whose absent components carry identity rows.  The embedding is
// exact for every grouping (the absent rows and columns are decoupled identities); the
// grouping only steers the aggregation.  Duplicate (I, J) triplets are summed.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <unordered_map>
#include <vector>

#include "mesh.h"
#include "sg_common.cuh"

namespace sg {

namespace {

struct IjvInstance {
    int device = 0;
    cudaStream_t stream = nullptr;
    int64_t n = 0;          // matrix size (free DOFs)
    int64_t nnz_in = 0;     // triplets per value array
    int b = 3, nns = 0;
    int64_t n_nodes = 0;
    sg_bsr bsr;
    double *d_vals = nullptr;            // block values, n_blocks * b * b
    double *d_V = nullptr;               // the caller's values, triplet order
    int64_t *d_order = nullptr;          // triplet indices sorted by value slot
    int64_t *d_seg_ptr = nullptr;        // segments of d_order with one slot each
    int64_t *d_seg_slot = nullptr;
    int64_t n_seg = 0;
    int64_t *d_ident = nullptr;          // diagonal slots of absent components (set to 1)
    int64_t n_ident = 0;
    int64_t *d_q2dof = nullptr;          // free DOF -> block DOF
    double *d_r = nullptr, *d_y = nullptr;      // n, free-DOF order
    double *d_rb = nullptr, *d_yb = nullptr;    // n_nodes * b, block order
    sg_amg *amg = nullptr;
    int64_t full_builds = 0, value_updates = 0;

    ~IjvInstance() {
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(device);
        if (amg) sg_amg_destroy(amg);
        cudaFree(d_vals); cudaFree(d_V); cudaFree(d_order); cudaFree(d_seg_ptr); cudaFree(d_seg_slot);
        cudaFree(d_ident); cudaFree(d_q2dof); cudaFree(d_r); cudaFree(d_y); cudaFree(d_rb); cudaFree(d_yb);
        bsr_free(bsr);
        if (stream) cudaStreamDestroy(stream);
        cudaSetDevice(cur);
    }
};

std::mutex g_mu;
std::unordered_map<std::string, std::unique_ptr<IjvInstance>> g_instances;

// vals[slot of segment u] = sum of V over the segment's triplets (fixed order: deterministic)
__global__ void k_ijv_scatter(int64_t n_seg, const int64_t *__restrict__ seg_ptr, const int64_t *__restrict__ seg_slot,
                              const int64_t *__restrict__ order, const double *__restrict__ V, double *__restrict__ vals) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n_seg; u += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int64_t p = seg_ptr[u]; p < seg_ptr[u + 1]; ++p) s += V[order[p]];
        vals[seg_slot[u]] = s;
    }
}

__global__ void k_ijv_identity(int64_t n, const int64_t *__restrict__ slots, double *__restrict__ vals) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        vals[slots[i]] = 1.0;
}

// block-order vector from a free-DOF-order one (absent components zero) and back
__global__ void k_ijv_to_blocks(int64_t n, const int64_t *__restrict__ q2dof, const double *__restrict__ r,
                                double *__restrict__ rb) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        rb[q2dof[q]] = r[q];
}

__global__ void k_ijv_from_blocks(int64_t n, const int64_t *__restrict__ q2dof, const double *__restrict__ yb,
                                  double *__restrict__ y) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        y[q] = yb[q2dof[q]];
}

template <typename T>
int upload_vec(T **dst, const std::vector<T> &v) {
    SG_CUDA(device_alloc(dst, sizeof(T) * std::max<size_t>(v.size(), 1)));
    if (!v.empty()) SG_CUDA(cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return SG_OK;
}

int load_values(IjvInstance &inst, const double *V) {
    const cudaStream_t st = inst.stream;
    const int64_t nv = inst.bsr.n_blocks * inst.b * inst.b;
    if (inst.nnz_in) SG_CUDA(cudaMemcpyAsync(inst.d_V, V, sizeof(double) * inst.nnz_in, cudaMemcpyHostToDevice, st));
    SG_CUDA(cudaMemsetAsync(inst.d_vals, 0, sizeof(double) * nv, st));
    if (inst.n_seg)
        k_ijv_scatter<<<grid_for(inst.n_seg, 256), 256, 0, st>>>(inst.n_seg, inst.d_seg_ptr, inst.d_seg_slot,
                                                                inst.d_order, inst.d_V, inst.d_vals);
    if (inst.n_ident) k_ijv_identity<<<grid_for(inst.n_ident, 256), 256, 0, st>>>(inst.n_ident, inst.d_ident, inst.d_vals);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

// Pattern, value map, block embedding and the AMG of a new instance.  Numeric options:
// [max_levels, coarse_size, cheb_degree, cheb_ratio, power_its, mixed, omega_scale, theta,
// fine_half] as for sg_amg_create.
int build_instance(IjvInstance &inst, const double *I, const double *J, const double *V, int64_t nnz, int64_t n,
                   const double *Z, int32_t nns, const double *dof_func, int32_t num_functions, const double *opts,
                   int32_t n_opts) {
    const int b = num_functions;
    inst.n = n;
    inst.nnz_in = nnz;
    inst.b = b;
    // components and nodes
    std::vector<int32_t> comp(n);
    for (int64_t q = 0; q < n; ++q) {
        const double c = dof_func ? dof_func[q] : (double)(q % b);
        const long long ci = std::llround(c);
        if (!(ci >= 0 && ci < b)) return set_error(SG_ERR_ARG, "dof_func values must lie in [0, num_functions - 1]");
        comp[q] = (int32_t)ci;
    }
    std::vector<int64_t> node(n);
    int64_t nn = 0;
    for (int64_t q = 0; q < n; ++q) {
        if (q == 0 || comp[q] <= comp[q - 1]) ++nn;
        node[q] = nn - 1;
    }
    inst.n_nodes = nn;
    if (nn > INT32_MAX) return set_error(SG_ERR_ARG, "too many nodes for 32-bit block indices");
    std::vector<int64_t> q2dof(n);
    std::vector<uint8_t> present((size_t)nn * b, 0);
    for (int64_t q = 0; q < n; ++q) {
        q2dof[q] = node[q] * b + comp[q];
        present[(size_t)q2dof[q]] = 1;
    }
    // triplets -> (block row, block column)
    std::vector<int64_t> gi(nnz), gj(nnz);
    for (int64_t k = 0; k < nnz; ++k) {
        const long long i = std::llround(I[k]) - 1, j = std::llround(J[k]) - 1;
        if (i < 0 || i >= n || j < 0 || j >= n) return set_error(SG_ERR_ARG, "I and J must lie in 1..n");
        gi[k] = i;
        gj[k] = j;
    }
    // block pattern: rows sorted, diagonal always present
    std::vector<int64_t> cnt(nn + 1, 0);
    for (int64_t k = 0; k < nnz; ++k) cnt[node[gi[k]] + 1]++;
    for (int64_t r = 0; r < nn; ++r) cnt[r + 1] += cnt[r] + 1;   // + the diagonal
    std::vector<int32_t> cols(cnt[nn]);
    {
        std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
        for (int64_t r = 0; r < nn; ++r) cols[fill[r]++] = (int32_t)r;
        for (int64_t k = 0; k < nnz; ++k) cols[fill[node[gi[k]]]++] = (int32_t)node[gj[k]];
    }
    sg_bsr &B = inst.bsr;
    B.b = b;
    B.n_rows = nn;
    B.row_ptr.assign(nn + 1, 0);
    B.col.clear();
    B.col.reserve(cols.size());
    for (int64_t r = 0; r < nn; ++r) {
        auto *s = cols.data() + cnt[r], *e = cols.data() + cnt[r + 1];
        std::sort(s, e);
        e = std::unique(s, e);
        B.col.insert(B.col.end(), s, e);
        if (B.col.size() > (size_t)INT32_MAX) return set_error(SG_ERR_ARG, "too many blocks for 32-bit indices");
        B.row_ptr[r + 1] = (int32_t)B.col.size();
    }
    std::vector<int32_t>().swap(cols);
    B.n_blocks = (int64_t)B.col.size();
    // value slot of every triplet, then the triplets sorted by slot (segments of equal slot)
    const int bb = b * b;
    std::vector<int64_t> slot(nnz);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nnz; ++k) {
        const int64_t r = node[gi[k]];
        const int32_t c = (int32_t)node[gj[k]];
        const int32_t *s = B.col.data() + B.row_ptr[r], *e = B.col.data() + B.row_ptr[r + 1];
        const int64_t blk = std::lower_bound(s, e, c) - B.col.data();
        slot[k] = blk * bb + comp[gi[k]] * b + comp[gj[k]];
    }
    std::vector<int64_t>().swap(gi);
    std::vector<int64_t>().swap(gj);
    std::vector<int64_t> order(nnz);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t c) { return slot[a] < slot[c]; });
    std::vector<int64_t> seg_ptr, seg_slot;
    seg_ptr.reserve(nnz + 1);
    seg_slot.reserve(nnz);
    for (int64_t p = 0; p < nnz; ++p) {
        if (p == 0 || slot[order[p]] != slot[order[p - 1]]) {
            seg_ptr.push_back(p);
            seg_slot.push_back(slot[order[p]]);
        }
    }
    seg_ptr.push_back(nnz);
    inst.n_seg = (int64_t)seg_slot.size();
    // identity on the diagonal of absent components
    std::vector<int64_t> ident;
    std::vector<int32_t> diag_blk(nn);
    for (int64_t r = 0; r < nn; ++r) {
        const int32_t *s = B.col.data() + B.row_ptr[r], *e = B.col.data() + B.row_ptr[r + 1];
        diag_blk[r] = (int32_t)(std::lower_bound(s, e, (int32_t)r) - B.col.data());
        for (int c = 0; c < b; ++c)
            if (!present[(size_t)r * b + c]) ident.push_back((int64_t)diag_blk[r] * bb + c * b + c);
    }
    inst.n_ident = (int64_t)ident.size();
    // device side
    int rc = bsr_upload(B);
    if (!rc) rc = upload_vec(&inst.d_order, order);
    if (!rc) rc = upload_vec(&inst.d_seg_ptr, seg_ptr);
    if (!rc) rc = upload_vec(&inst.d_seg_slot, seg_slot);
    if (!rc) rc = upload_vec(&inst.d_ident, ident);
    if (!rc) rc = upload_vec(&inst.d_q2dof, q2dof);
    if (rc) return rc;
    const int64_t nd = nn * b;
    SG_CUDA(device_alloc(&inst.d_vals, sizeof(double) * std::max<int64_t>(B.n_blocks * bb, 1)));
    SG_CUDA(device_alloc(&inst.d_V, sizeof(double) * std::max<int64_t>(nnz, 1)));
    SG_CUDA(device_alloc(&inst.d_r, sizeof(double) * n));
    SG_CUDA(device_alloc(&inst.d_y, sizeof(double) * n));
    SG_CUDA(device_alloc(&inst.d_rb, sizeof(double) * nd));
    SG_CUDA(device_alloc(&inst.d_yb, sizeof(double) * nd));
    SG_CUDA(cudaMemsetAsync(inst.d_rb, 0, sizeof(double) * nd, inst.stream));
    rc = load_values(inst, V);
    if (rc) return rc;
    // near-null space in block order (column-major, zero on absent components); without Z,
    // the b translations
    const int k = (Z && nns > 0) ? nns : b;
    inst.nns = k;
    std::vector<double> Zb((size_t)nd * k, 0.0);
    for (int c = 0; c < k; ++c)
        for (int64_t q = 0; q < n; ++q)
            Zb[(size_t)c * nd + q2dof[q]] = (Z && nns > 0) ? Z[(size_t)c * n + q] : (comp[q] == c ? 1.0 : 0.0);
    std::vector<uint8_t> fixed(nd);
    for (int64_t d = 0; d < nd; ++d) fixed[d] = present[d] ? 0 : 1;
    rc = sg_amg_create(&inst.bsr, inst.d_vals, Zb.data(), k, fixed.data(), opts, n_opts, &inst.amg, inst.stream);
    if (!rc) rc = sg_amg_update(inst.amg, inst.d_vals, inst.stream);
    if (!rc) SG_CUDA(cudaStreamSynchronize(inst.stream));
    return rc;
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

IjvInstance *find(const char *id) {
    if (!id) return nullptr;
    auto it = g_instances.find(id);
    return it == g_instances.end() ? nullptr : it->second.get();
}

struct DeviceScope {
    int saved = 0;
    explicit DeviceScope(int dev) {
        cudaGetDevice(&saved);
        cudaSetDevice(dev);
    }
    ~DeviceScope() { cudaSetDevice(saved); }
};

}  // namespace
}  // namespace sg

using namespace sg;

extern "C" int sg_amg_setup_ijv(const char *id, const double *I, const double *J, const double *V, int64_t nnz,
                                int64_t n, const double *Z, int32_t nns, const double *dof_func,
                                int32_t num_functions, const double *opts, int32_t n_opts, int32_t force_rebuild,
                                double *setup_seconds) {
    SG_CHECK_ARG(id && id[0], "empty instance id");
    SG_CHECK_ARG(nnz >= 0 && n > 0, "n must be positive and nnz non-negative");
    SG_CHECK_ARG(nnz == 0 || (I && J && V), "null I, J or V");
    SG_CHECK_ARG(num_functions >= 1 && num_functions <= 3,
                 "num_functions must be 1, 2 or 3 (the AMG works on 1 x 1, 2 x 2 or 3 x 3 node blocks)");
    SG_CHECK_ARG(nns >= 0 && nns <= 6 && (nns == 0 || Z), "near-null space: 0..6 columns, non-null when given");
    SG_CHECK_ARG(nns == 0 || (num_functions == 3 && (nns == 6 || nns == 3)) || (num_functions == 2 && nns == 3) ||
                     (num_functions == 1 && nns == 1),
                 "near-null space dimension: 6 or 3 for 3 functions, 3 for 2 functions, 1 for 1 function");
    SG_CHECK_ARG(!(num_functions == 2 && nns == 0), "2 functions need the 3 rigid-body modes (Z)");
    std::lock_guard<std::mutex> lock(g_mu);
    const auto t0 = std::chrono::steady_clock::now();
    IjvInstance *old = find(id);
    if (old && !force_rebuild && nnz == old->nnz_in) {
        // pattern kept: new values, numeric set-up
        DeviceScope ds(old->device);
        int rc = load_values(*old, V);
        if (!rc) rc = sg_amg_update(old->amg, old->d_vals, old->stream);
        if (!rc) SG_CUDA(cudaStreamSynchronize(old->stream));
        if (rc) return rc;
        old->value_updates++;
        if (setup_seconds) *setup_seconds = seconds_since(t0);
        return SG_OK;
    }
    if (old) g_instances.erase(id);
    auto inst = std::make_unique<IjvInstance>();
    SG_CUDA(cudaGetDevice(&inst->device));
    SG_CUDA(cudaStreamCreateWithFlags(&inst->stream, cudaStreamNonBlocking));
    const int rc = build_instance(*inst, I, J, V, nnz, n, Z, nns, dof_func, num_functions, opts, n_opts);
    if (rc) return rc;
    inst->full_builds = 1;
    if (setup_seconds) *setup_seconds = seconds_since(t0);
    g_instances[id] = std::move(inst);
    return SG_OK;
}

extern "C" int sg_amg_update_values(const char *id, const double *V, int64_t nnz, double *setup_seconds) {
    SG_CHECK_ARG(id, "null instance id");
    std::lock_guard<std::mutex> lock(g_mu);
    IjvInstance *inst = find(id);
    if (!inst) return set_error(SG_ERR_STATE, "unknown instance id: call sg_amg_setup_ijv first");
    SG_CHECK_ARG(nnz == inst->nnz_in, "V length must match the triplet count of sg_amg_setup_ijv");
    SG_CHECK_ARG(nnz == 0 || V, "null V");
    const auto t0 = std::chrono::steady_clock::now();
    DeviceScope ds(inst->device);
    int rc = load_values(*inst, V);
    if (!rc) rc = sg_amg_update(inst->amg, inst->d_vals, inst->stream);
    if (!rc) SG_CUDA(cudaStreamSynchronize(inst->stream));
    if (rc) return rc;
    inst->value_updates++;
    if (setup_seconds) *setup_seconds = seconds_since(t0);
    return SG_OK;
}

extern "C" int sg_amg_apply_host(const char *id, const double *r, double *y, int64_t n) {
    SG_CHECK_ARG(id && r && y, "null argument");
    std::lock_guard<std::mutex> lock(g_mu);
    IjvInstance *inst = find(id);
    if (!inst) return set_error(SG_ERR_STATE, "unknown instance id: call sg_amg_setup_ijv first");
    SG_CHECK_ARG(n == inst->n, "vector length does not match the preconditioner size");
    DeviceScope ds(inst->device);
    const cudaStream_t st = inst->stream;
    SG_CUDA(cudaMemcpyAsync(inst->d_r, r, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    k_ijv_to_blocks<<<grid_for(n, 256), 256, 0, st>>>(n, inst->d_q2dof, inst->d_r, inst->d_rb);
    SG_CUDA(cudaGetLastError());
    int rc = sg_amg_apply(inst->amg, inst->d_rb, inst->d_yb, st);
    if (rc) return rc;
    k_ijv_from_blocks<<<grid_for(n, 256), 256, 0, st>>>(n, inst->d_q2dof, inst->d_yb, inst->d_y);
    SG_CUDA(cudaGetLastError());
    SG_CUDA(cudaMemcpyAsync(y, inst->d_y, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    return SG_OK;
}

extern "C" int sg_amg_clear(const char *id) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!id) {
        g_instances.clear();
        return SG_OK;
    }
    g_instances.erase(id);
    return SG_OK;
}

extern "C" int sg_amg_ijv_info(const char *id, int64_t *info, int32_t cap) {
    SG_CHECK_ARG(info && cap >= 1, "bad argument");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!id) {
        info[0] = (int64_t)g_instances.size();
        return SG_OK;
    }
    IjvInstance *inst = find(id);
    if (!inst) return set_error(SG_ERR_STATE, "unknown instance id");
    const int64_t v[] = {inst->n, inst->nnz_in, inst->b, inst->nns, inst->n_nodes, inst->bsr.n_blocks,
                         inst->full_builds, inst->value_updates};
    for (int i = 0; i < cap && i < 8; ++i) info[i] = v[i];
    return SG_OK;
}
