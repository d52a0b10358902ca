// Device-resident mesh data and sparsity patterns (internal header).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

// Block-sparse (BSR) pattern with square b x b blocks, block-row CSR indexing.  Values live
// in caller-owned arrays of n_blocks * b * b entries, row-major inside each block.
struct sg_bsr {
    int b = 3;
    int64_t n_rows = 0;     // block rows (== block columns)
    int64_t n_blocks = 0;
    std::vector<int32_t> row_ptr, col;   // host copy
    int32_t *d_row_ptr = nullptr, *d_col = nullptr;
    int32_t *d_diag = nullptr;           // block index of the diagonal block of each row
    int32_t *d_transpose = nullptr;      // block index of block (j, i) for block (i, j)
    int32_t *d_row_of = nullptr;         // block row of every block
    int owned_by_mesh = 0;
};

struct sg_mesh {
    int dim = 3, np = 10, nq = 11, ns = 6;
    int64_t n_n = 0, n_e = 0, n_int = 0;
    std::vector<int32_t> elem;        // element-major: elem[e * np + i], 0-based
    std::vector<uint8_t> Q;           // node-major: Q[node * dim + comp]
    std::vector<int64_t> dof2q;       // dof -> free index, -1 if Dirichlet
    int64_t n_Q = 0, nnz_ref = 0;
    sg_bsr bsr;                       // node adjacency, b = dim
    // the same node adjacency with 1 x 1 blocks for scalar (pore-pressure) systems: device
    // arrays shared with bsr (not freed through bsr1), host copies made on first request
    sg_bsr bsr1;
    bool bsr1_ready = false;
    // device
    int32_t *d_elem = nullptr;        // n_e * np
    double *d_dphi = nullptr;         // n_int * dim * np, per point [d][i]
    double *d_w = nullptr;            // n_int
    double *d_mask = nullptr;         // dim * n_n, 1 free / 0 Dirichlet
    int32_t *d_pair_blk = nullptr;    // n_e * np * np: block index of (node_i, node_j)
    int64_t *d_ref2bsr = nullptr;     // nnz_ref: value index of K(ref_I, ref_J) inside BSR values
    // deterministic assembly of P2 tetrahedra: every BSR block's contributions (element e,
    // upper node-block slot s of that element, transposed flag in bit 31) in element order
    int32_t *d_contrib_ptr = nullptr; // n_blocks + 1
    uint32_t *d_contrib = nullptr;    // n_e * np * np entries: e * 55 + s | transposed << 31
    double *d_ke = nullptr;           // n_e * 55 * 10: element upper node blocks, 9 values + 1 pad (allocated on first use)
    int device = 0;
};

namespace sg {
int bsr_upload(sg_bsr &m);
void bsr_free(sg_bsr &m);
}  // namespace sg
