// Mesh object: host construction of the sparsity patterns and upload of element data.
//
// Pattern facts used here (checked against a literal restatement of
// +CONSTITUTIVE_PROBLEM/CONSTITUTIVE.m:393-464 in the tests): the maximal symbolic pattern of
// K(Q,Q) = spones(B_Q)' spones(D) spones(B_Q) is the node adjacency (nodes sharing an
// element) expanded to dim x dim blocks and restricted to free DOFs, because every P2 basis
// gradient is non-zero at some quadrature point of each element and D is a full block.
// Octave's find() lists it column by column; for a symmetric pattern that is the row-major
// (CSR) order with the roles of I and J swapped, which is how it is enumerated here.
//
// Device layouts:
//   d_elem     [e][i]                 int32, 0-based node ids
//   d_dphi     [g][d][i]              physical basis gradients per point (g = e*nq + q)
//   d_w        [g]                    quadrature weights |det J| * w_q
//   d_mask     [node*dim + comp]      1.0 free, 0.0 Dirichlet
//   BSR        node adjacency, dim x dim blocks, row-major inside a block
//   d_pair_blk [e][i][j]              BSR block of (node_i, node_j)
#include <omp.h>

#include <algorithm>
#include <cstring>
#include <new>

#include "mesh.h"
#include "sg_common.cuh"

namespace sg {

template <typename T>
static int upload(T **dst, const T *src, size_t n) {
    if (n == 0) { *dst = nullptr; return SG_OK; }
    SG_CUDA(sg::device_alloc((void **)dst, n * sizeof(T)));
    SG_CUDA(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
    return SG_OK;
}

int bsr_upload(sg_bsr &m) {
    const int64_t nr = m.n_rows, nb = m.n_blocks;
    std::vector<int32_t> diag(nr, -1), tr(nb, -1), row_of(nb);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < nr; ++i) {
        const int32_t *b = m.col.data() + m.row_ptr[i], *e = m.col.data() + m.row_ptr[i + 1];
        const int32_t *d = std::lower_bound(b, e, (int32_t)i);
        if (d != e && *d == i) diag[i] = (int32_t)(d - m.col.data());
        for (int32_t p = m.row_ptr[i]; p < m.row_ptr[i + 1]; ++p) {
            row_of[p] = (int32_t)i;
            const int32_t j = m.col[p];
            const int32_t *bj = m.col.data() + m.row_ptr[j], *ej = m.col.data() + m.row_ptr[j + 1];
            const int32_t *t = std::lower_bound(bj, ej, (int32_t)i);
            if (t != ej && *t == i) tr[p] = (int32_t)(t - m.col.data());
        }
    }
    int rc = upload(&m.d_row_ptr, m.row_ptr.data(), nr + 1);
    if (!rc) rc = upload(&m.d_col, m.col.data(), nb);
    if (!rc) rc = upload(&m.d_diag, diag.data(), nr);
    if (!rc) rc = upload(&m.d_transpose, tr.data(), nb);
    if (!rc) rc = upload(&m.d_row_of, row_of.data(), nb);
    return rc;
}

void bsr_free(sg_bsr &m) {
    cudaFree(m.d_row_ptr);
    cudaFree(m.d_col);
    cudaFree(m.d_diag);
    cudaFree(m.d_transpose);
    cudaFree(m.d_row_of);
    m.d_row_ptr = m.d_col = m.d_diag = m.d_transpose = m.d_row_of = nullptr;
}

// Node adjacency (nodes sharing an element), sorted rows, including the diagonal.
static void node_adjacency(const std::vector<int32_t> &elem, int np, int64_t n_n, int64_t n_e,
                           std::vector<int32_t> &row_ptr, std::vector<int32_t> &col) {
    std::vector<int64_t> inc_ptr(n_n + 1, 0);
    for (int64_t k = 0; k < n_e * np; ++k) inc_ptr[elem[k] + 1]++;
    for (int64_t i = 0; i < n_n; ++i) inc_ptr[i + 1] += inc_ptr[i];
    std::vector<int64_t> inc(n_e * np), fill(inc_ptr.begin(), inc_ptr.end() - 1);
    for (int64_t e = 0; e < n_e; ++e)
        for (int i = 0; i < np; ++i) inc[fill[elem[e * np + i]]++] = e;
    std::vector<int32_t> cnt(n_n, 0);
    std::vector<std::vector<int32_t>> rows(n_n);
#pragma omp parallel for schedule(dynamic, 512)
    for (int64_t v = 0; v < n_n; ++v) {
        std::vector<int32_t> &r = rows[v];
        r.reserve((inc_ptr[v + 1] - inc_ptr[v]) * np);
        for (int64_t k = inc_ptr[v]; k < inc_ptr[v + 1]; ++k) {
            const int64_t e = inc[k];
            for (int i = 0; i < np; ++i) r.push_back(elem[e * np + i]);
        }
        std::sort(r.begin(), r.end());
        r.erase(std::unique(r.begin(), r.end()), r.end());
        cnt[v] = (int32_t)r.size();
    }
    row_ptr.assign(n_n + 1, 0);
    for (int64_t v = 0; v < n_n; ++v) row_ptr[v + 1] = row_ptr[v] + cnt[v];
    col.resize(row_ptr[n_n]);
#pragma omp parallel for schedule(dynamic, 512)
    for (int64_t v = 0; v < n_n; ++v) {
        std::copy(rows[v].begin(), rows[v].end(), col.begin() + row_ptr[v]);
        std::vector<int32_t>().swap(rows[v]);
    }
}

static int mesh_build(sg_mesh *m, const int32_t *elem, const double *D1, const double *D2, const double *D3,
                      const double *W, const uint8_t *Q) {
    const int dim = m->dim, np = m->np;
    const int64_t n_n = m->n_n, n_e = m->n_e, n_int = m->n_int;
    m->elem.assign(elem, elem + n_e * np);
    for (int64_t k = 0; k < n_e * np; ++k)
        if (m->elem[k] < 0 || m->elem[k] >= n_n) return set_error(SG_ERR_ARG, "element node index out of range");
    m->Q.assign(Q, Q + n_n * dim);
    m->dof2q.assign(n_n * dim, -1);
    int64_t q = 0;
    for (int64_t d = 0; d < n_n * dim; ++d)
        if (m->Q[d]) m->dof2q[d] = q++;
    m->n_Q = q;

    sg_bsr &B = m->bsr;
    B.b = dim;
    B.n_rows = n_n;
    node_adjacency(m->elem, np, n_n, n_e, B.row_ptr, B.col);
    B.n_blocks = B.row_ptr[n_n];
    B.owned_by_mesh = 1;

    // nnz of K(Q,Q): every free row of node I has the same columns
    std::vector<int32_t> nfree(n_n);
    for (int64_t v = 0; v < n_n; ++v) {
        int c = 0;
        for (int k = 0; k < dim; ++k) c += m->Q[v * dim + k] ? 1 : 0;
        nfree[v] = c;
    }
    int64_t nnz = 0;
    for (int64_t v = 0; v < n_n; ++v) {
        if (!nfree[v]) continue;
        int64_t rowlen = 0;
        for (int32_t p = B.row_ptr[v]; p < B.row_ptr[v + 1]; ++p) rowlen += nfree[B.col[p]];
        nnz += rowlen * nfree[v];
    }
    m->nnz_ref = nnz;

    // element pair -> BSR block
    std::vector<int32_t> pair((size_t)n_e * np * np);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n_e; ++e) {
        for (int i = 0; i < np; ++i) {
            const int32_t a = m->elem[e * np + i];
            const int32_t *b0 = B.col.data() + B.row_ptr[a], *b1 = B.col.data() + B.row_ptr[a + 1];
            for (int j = 0; j < np; ++j) {
                const int32_t c = m->elem[e * np + j];
                pair[(e * np + i) * np + j] = (int32_t)(std::lower_bound(b0, b1, c) - B.col.data());
            }
        }
    }
    // per-point gradients, interleaved [g][d][i]
    std::vector<double> dphi((size_t)n_int * dim * np);
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < n_int; ++g) {
        for (int i = 0; i < np; ++i) {
            dphi[(g * dim + 0) * np + i] = D1[g * np + i];
            dphi[(g * dim + 1) * np + i] = D2[g * np + i];
            if (dim == 3) dphi[(g * dim + 2) * np + i] = D3[g * np + i];
        }
    }
    std::vector<double> mask(n_n * dim);
    for (int64_t d = 0; d < n_n * dim; ++d) mask[d] = m->Q[d] ? 1.0 : 0.0;

    // contribution lists of the deterministic P2-tetrahedron assembly: block (node_i, node_j)
    // of element e takes its upper slot s(min(i,j), max(i,j)), transposed when i > j; the lists
    // are filled in element order, so every block sums its contributions in a fixed order
    std::vector<int32_t> cptr;
    std::vector<uint32_t> contrib;
    if (dim == 3 && np == 10 && n_e * 55 < ((int64_t)1 << 31)) {
        cptr.assign(B.n_blocks + 1, 0);
        for (size_t t = 0; t < pair.size(); ++t) cptr[pair[t] + 1]++;
        for (int64_t p = 0; p < B.n_blocks; ++p) cptr[p + 1] += cptr[p];
        std::vector<int32_t> fill(cptr.begin(), cptr.end() - 1);
        contrib.resize(pair.size());
        for (int64_t e = 0; e < n_e; ++e)
            for (int i = 0; i < np; ++i)
                for (int j = 0; j < np; ++j) {
                    const int lo = std::min(i, j), hi = std::max(i, j);
                    const uint32_t slot = (uint32_t)(lo * np - lo * (lo - 1) / 2 + (hi - lo));
                    contrib[fill[pair[(e * np + i) * np + j]]++] =
                        (uint32_t)(e * 55 + slot) | (i > j ? 0x80000000u : 0u);
                }
    }

    int rc = bsr_upload(B);
    if (!rc && !contrib.empty()) rc = upload(&m->d_contrib_ptr, cptr.data(), cptr.size());
    if (!rc && !contrib.empty()) rc = upload(&m->d_contrib, contrib.data(), contrib.size());
    if (!rc) rc = upload(&m->d_elem, m->elem.data(), (size_t)n_e * np);
    if (!rc) rc = upload(&m->d_dphi, dphi.data(), dphi.size());
    if (!rc) rc = upload(&m->d_w, W, (size_t)n_int);
    if (!rc) rc = upload(&m->d_mask, mask.data(), mask.size());
    if (!rc) rc = upload(&m->d_pair_blk, pair.data(), pair.size());
    return rc;
}

// Reference-order enumeration helpers ------------------------------------------------

// For every free row q (in order) visit its entries in order: f(k, qrow, qcol, block p, a, b)
template <typename F>
static void for_each_ref_entry(const sg_mesh *m, F f) {
    const int dim = m->dim;
    const sg_bsr &B = m->bsr;
    int64_t k = 0;
    for (int64_t v = 0; v < m->n_n; ++v) {
        for (int a = 0; a < dim; ++a) {
            const int64_t qr = m->dof2q[v * dim + a];
            if (qr < 0) continue;
            for (int32_t p = B.row_ptr[v]; p < B.row_ptr[v + 1]; ++p) {
                const int32_t w = B.col[p];
                for (int b = 0; b < dim; ++b) {
                    const int64_t qc = m->dof2q[(int64_t)w * dim + b];
                    if (qc < 0) continue;
                    f(k++, qr, qc, p, a, b);
                }
            }
        }
    }
}

}  // namespace sg

using namespace sg;

extern "C" int sg_mesh_create(int dim, int32_t n_p, int32_t n_q, int64_t n_n, int64_t n_e, const int32_t *elem,
                              const double *DPhi1, const double *DPhi2, const double *DPhi3, const double *weight,
                              const uint8_t *Q, sg_mesh **out) {
    SG_CHECK_ARG(out, "null output handle");
    *out = nullptr;
    SG_CHECK_ARG(dim == 2 || dim == 3, "dim must be 2 or 3");
    SG_CHECK_ARG(n_p > 0 && n_p <= 20 && n_q > 0 && n_q <= 32, "n_p must be 1..20 and n_q 1..32");
    SG_CHECK_ARG(n_n > 0 && n_e > 0 && n_n < (1ll << 31) / 4, "bad node/element counts");
    SG_CHECK_ARG(elem && DPhi1 && DPhi2 && weight && Q && (dim == 2 || DPhi3), "null input pointer");
    sg_mesh *m = new (std::nothrow) sg_mesh();
    if (!m) return set_error(SG_ERR_NOMEM, "host allocation");
    m->dim = dim;
    m->np = n_p;
    m->nq = n_q;
    m->ns = dim == 3 ? 6 : 3;
    m->n_n = n_n;
    m->n_e = n_e;
    m->n_int = n_e * n_q;
    cudaGetDevice(&m->device);
    int rc = mesh_build(m, elem, DPhi1, DPhi2, DPhi3, weight, Q);
    if (rc) {
        sg_mesh_destroy(m);
        return rc;
    }
    if (m->bsr.n_blocks >= (1ll << 31) / 9) {
        sg_mesh_destroy(m);
        return set_error(SG_ERR_ARG, "pattern too large for 32-bit value indexing");
    }
    *out = m;
    return SG_OK;
}

extern "C" int sg_mesh_destroy(sg_mesh *m) {
    if (!m) return SG_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(m->device);
    bsr_free(m->bsr);
    cudaFree(m->d_elem);
    cudaFree(m->d_dphi);
    cudaFree(m->d_w);
    cudaFree(m->d_mask);
    cudaFree(m->d_pair_blk);
    cudaFree(m->d_contrib_ptr);
    cudaFree(m->d_contrib);
    cudaFree(m->d_ke);
    cudaFree(m->d_ref2bsr);
    cudaSetDevice(cur);
    delete m;
    return SG_OK;
}

extern "C" int sg_mesh_sizes(const sg_mesh *m, int64_t *sizes) {
    SG_CHECK_ARG(m && sizes, "null argument");
    sizes[0] = m->n_n * m->dim;
    sizes[1] = m->n_Q;
    sizes[2] = m->nnz_ref;
    sizes[3] = m->bsr.n_blocks;
    sizes[4] = m->n_int;
    return SG_OK;
}

extern "C" int sg_mesh_bsr(const sg_mesh *m, const sg_bsr **bsr) {
    SG_CHECK_ARG(m && bsr, "null argument");
    *bsr = &m->bsr;
    return SG_OK;
}

extern "C" int sg_mesh_pattern(const sg_mesh *m, int64_t *ref_I, int64_t *ref_J, int64_t *transpose_perm) {
    SG_CHECK_ARG(m, "null mesh");
    if (ref_I || ref_J) {
        for_each_ref_entry(m, [&](int64_t k, int64_t qr, int64_t qc, int32_t, int, int) {
            if (ref_I) ref_I[k] = qc + 1;
            if (ref_J) ref_J[k] = qr + 1;
        });
    }
    if (transpose_perm) {
        // row start of every free row, then position of (qc, qr) within row qc
        std::vector<int64_t> rstart(m->n_Q + 1, 0);
        std::vector<int64_t> first_col;  // not needed: columns within a row are sorted
        const int dim = m->dim;
        const sg_bsr &B = m->bsr;
        std::vector<int32_t> blk_off(B.n_blocks);
        std::vector<int32_t> nfree(m->n_n);
        for (int64_t v = 0; v < m->n_n; ++v) {
            int c = 0;
            for (int k = 0; k < dim; ++k) c += m->Q[v * dim + k] ? 1 : 0;
            nfree[v] = c;
        }
        for (int64_t v = 0; v < m->n_n; ++v) {
            int32_t off = 0;
            for (int32_t p = B.row_ptr[v]; p < B.row_ptr[v + 1]; ++p) {
                blk_off[p] = off;
                off += nfree[B.col[p]];
            }
        }
        int64_t k = 0;
        std::vector<int64_t> rowstart_of_q(m->n_Q);
        for (int64_t v = 0; v < m->n_n; ++v) {
            int64_t rowlen = 0;
            for (int32_t p = B.row_ptr[v]; p < B.row_ptr[v + 1]; ++p) rowlen += nfree[B.col[p]];
            for (int a = 0; a < dim; ++a) {
                const int64_t q = m->dof2q[v * dim + a];
                if (q < 0) continue;
                rowstart_of_q[q] = k;
                k += rowlen;
            }
        }
        auto rank = [&](int64_t node, int b) {
            int r = 0;
            for (int t = 0; t < b; ++t) r += m->Q[node * dim + t] ? 1 : 0;
            return r;
        };
        std::vector<int32_t> blkT(B.n_blocks);
        cudaMemcpy(blkT.data(), B.d_transpose, sizeof(int32_t) * B.n_blocks, cudaMemcpyDeviceToHost);
        std::vector<int32_t> row_of_blk(B.n_blocks);
        for (int64_t v = 0; v < m->n_n; ++v)
            for (int32_t p = B.row_ptr[v]; p < B.row_ptr[v + 1]; ++p) row_of_blk[p] = (int32_t)v;
        for_each_ref_entry(m, [&](int64_t kk, int64_t, int64_t qc, int32_t p, int a, int) {
            // transposed entry lives in free row qc, block (J, I) = blkT[p], column comp a of node I
            const int32_t pt = blkT[p];
            const int64_t nodeI = row_of_blk[p];
            transpose_perm[kk] = rowstart_of_q[qc] + blk_off[pt] + rank(nodeI, a) + 1;
        });
    }
    return SG_OK;
}

extern "C" int sg_mesh_scatter_map(const sg_mesh *m, int64_t *smap) {
    SG_CHECK_ARG(m && smap, "null argument");
    const int dim = m->dim, np = m->np, nl = dim * np;
    const sg_bsr &B = m->bsr;
    std::vector<int32_t> nfree(m->n_n), blk_off(B.n_blocks);
    for (int64_t v = 0; v < m->n_n; ++v) {
        int c = 0;
        for (int k = 0; k < dim; ++k) c += m->Q[v * dim + k] ? 1 : 0;
        nfree[v] = c;
    }
    std::vector<int64_t> rowstart_of_q(m->n_Q);
    int64_t k = 0;
    for (int64_t v = 0; v < m->n_n; ++v) {
        int32_t off = 0;
        for (int32_t p = B.row_ptr[v]; p < B.row_ptr[v + 1]; ++p) {
            blk_off[p] = off;
            off += nfree[B.col[p]];
        }
        for (int a = 0; a < dim; ++a) {
            const int64_t q = m->dof2q[v * dim + a];
            if (q < 0) continue;
            rowstart_of_q[q] = k;
            k += off;
        }
    }
    std::vector<int32_t> pair((size_t)m->n_e * np * np);
    cudaMemcpy(pair.data(), m->d_pair_blk, sizeof(int32_t) * pair.size(), cudaMemcpyDeviceToHost);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < m->n_e; ++e) {
        int64_t *out = smap + e * (int64_t)nl * nl;
        for (int jj = 0; jj < nl; ++jj) {
            const int j = jj / dim, b = jj % dim;              // ref_J = dof(jj) -> CSR row
            const int64_t qr = m->dof2q[(int64_t)m->elem[e * np + j] * dim + b];
            for (int ii = 0; ii < nl; ++ii) {
                const int i = ii / dim, a = ii % dim;          // ref_I = dof(ii) -> CSR column
                const int64_t node_i = m->elem[e * np + i];
                const int64_t qc = m->dof2q[node_i * dim + a];
                int64_t val = 0;
                if (qr >= 0 && qc >= 0) {
                    const int32_t p = pair[(e * np + j) * np + i];   // block (node_j, node_i)
                    int r = 0;
                    for (int t = 0; t < a; ++t) r += m->Q[node_i * dim + t] ? 1 : 0;
                    val = rowstart_of_q[qr] + blk_off[p] + r + 1;
                }
                out[ii + (int64_t)nl * jj] = val;
            }
        }
    }
    return SG_OK;
}

extern "C" int sg_mesh_free_dofs(const sg_mesh *m, int64_t *q_flat) {
    SG_CHECK_ARG(m && q_flat, "null argument");
    for (int64_t d = 0; d < m->n_n * m->dim; ++d)
        if (m->dof2q[d] >= 0) q_flat[m->dof2q[d]] = d;
    return SG_OK;
}
