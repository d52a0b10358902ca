// Learned node-wise correction of the AMG V-cycle (no counterpart in the reference: the
// reference preconditions DFGMRES with one BoomerAMG V-cycle only,
// +LINEAR_SOLVERS/mex/hypre_boomeramg_mex.cpp:751-796).
//
// After the V-cycle z = V(r), the correction adds one learned block-Jacobi step on the
// fine level:
//
//     z  <-  z + C (r - A z),      C_i = M_i G_i D_i^{-1}          (per node i, 3 x 3)
//
// where D_i is the node's 3 x 3 diagonal block of A, M_i zeroes Dirichlet components and
// G_i = MLP(phi_i) is the output of a per-node network (16 -> 64 -> 64 -> 9, ReLU) evaluated
// once per matrix on node features phi (log diagonal, plastic fraction, coordinates,
// Dirichlet flag, Newton residual, strength ratio).  The correction is linear in r, so the
// preconditioner is a fixed linear operator for each matrix; the network only chooses the
// node-wise weights.  With the last layer at zero it is exactly the plain V-cycle.
//
// Training runs on vectors that the plain solver itself produced (residual sequences of the
// Newton system), rz_s = v_s - A V(v_s), d_s = M G (D^{-1} rz_s), e_s = rz_s - A d_s.  The
// default objective is the FP64 residual, L = (1/S) sum_s |e_s|^2 / |rz_s|^2 with
// dL/dG_i = (1/S) sum_s (-2/|rz_s|^2) (M A e_s)_i (D^{-1} rz_s)_i^T.  The alternative is the
// energy norm of the error the corrected cycle leaves: with
// A err_s = rz_s,  |err_s - d_s|_A^2 - |err_s|_A^2 = d_s' A d_s - 2 d_s' rz_s, so
//
//     L = (1/S) sum_s (d_s' A d_s - 2 d_s' rz_s) / (rz_s' D^{-1} rz_s),
//     dL/dG_i = (1/S) sum_s (-2 / rz_s' D^{-1} rz_s) (M e_s)_i (D^{-1} rz_s)_i^T
//
// (measured: it over-corrects the smooth error components and raises the FGMRES iteration
// counts several-fold, so it is kept as an option only).  The network runs on the tensor cores: BF16 operands staged in shared
// memory in the canonical no-swizzle K-major layout, tcgen05.mma with FP32 accumulators in
// tensor memory, one elected thread issuing, completion through an mbarrier; the backward
// pass recomputes the forward for each 128-node tile and accumulates the weight gradients
// in tensor memory across the tiles a CTA owns.  Every wait on the mbarrier is bounded; a
// wait that runs out sets the error flag, the CTA stops issuing, waits (bounded) once more
// for what it issued, frees its tensor memory and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include "mesh.h"
#include "sg_common.cuh"

extern "C" int sg_amg_apply(sg_amg *h, const double *r, double *z, void *stream);
extern "C" int sg_amg_set_correction(sg_amg *h, const double *C, void *stream);
extern "C" int sg_bsr_spmv_dev(const sg_bsr *A, const double *vals, const double *x, double *y, void *stream);
extern "C" int sg_dot_dev(int64_t n, const double *x, const double *y, double *result, void *stream);

namespace sg {
namespace lc {

constexpr int NF = 16;     // input features per node
constexpr int NH = 64;     // hidden width
constexpr int NO = 16;     // output columns (the first 9 are G, row-major 3 x 3)
constexpr int TILE = 128;  // nodes per tile (MMA M)
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + NF * NH;
constexpr int OFF_W2 = OFF_B1 + NH;
constexpr int OFF_B2 = OFF_W2 + NH * NH;
constexpr int OFF_W3 = OFF_B2 + NH;
constexpr int OFF_B3 = OFF_W3 + NH * NO;
constexpr int NPARAM = OFF_B3 + NO;   // 6288 (SG_LEARNED_NPARAM)

// shared-memory carve (bytes); every operand tile is in the canonical K-major layout
constexpr uint32_t S_W1T = 0;                      // B, N=64 (out) x K=16 (in)
constexpr uint32_t S_W2T = S_W1T + 64 * 16 * 2;    // B, N=64 x K=64
constexpr uint32_t S_W3T = S_W2T + 64 * 64 * 2;    // B, N=16 x K=64
constexpr uint32_t S_W3N = S_W3T + 16 * 64 * 2;    // B, N=64 (hidden) x K=16 (out)
constexpr uint32_t S_W2N = S_W3N + 64 * 16 * 2;    // B, N=64 (in) x K=64 (out)
constexpr uint32_t S_X = S_W2N + 64 * 64 * 2;      // A, 128 nodes x K=16
constexpr uint32_t S_XT = S_X + 128 * 16 * 2;      // B, N=16 features x K=128 nodes
constexpr uint32_t S_H1 = S_XT + 16 * 128 * 2;     // A, 128 x K=64
constexpr uint32_t S_H1T = S_H1 + 128 * 64 * 2;    // B, N=64 x K=128 nodes
constexpr uint32_t S_H2 = S_H1T + 64 * 128 * 2;    // A, 128 x K=64
constexpr uint32_t S_H2T = S_H2 + 128 * 64 * 2;    // A, M=128 (64 used) x K=128 nodes
constexpr uint32_t S_DY3 = S_H2T + 128 * 128 * 2;  // A, 128 x K=16
constexpr uint32_t S_DY3T = S_DY3 + 128 * 16 * 2;  // B, N=16 x K=128 nodes
constexpr uint32_t S_DZ2 = S_DY3T + 16 * 128 * 2;  // A, 128 x K=64
constexpr uint32_t S_DZ2T = S_DZ2 + 128 * 64 * 2;  // A, M=128 (64 used) x K=128 nodes
constexpr uint32_t S_DZ1T = S_DZ2T + 128 * 128 * 2;
constexpr uint32_t S_BIAS = S_DZ1T + 128 * 128 * 2;   // b1, b2, b3 (FP32)
constexpr uint32_t S_DB = S_BIAS + (NH + NH + NO) * 4; // bias-gradient sums per warp (FP32, 4 x 144)
constexpr uint32_t S_BAR = S_DB + 4 * (NH + NH + NO) * 4;
constexpr uint32_t S_TMEM = S_BAR + 8;
constexpr uint32_t SMEM_BYTES = S_TMEM + 8;
static_assert(SMEM_BYTES <= 227 * 1024, "shared memory carve too large");

// tensor-memory columns (FP32 accumulators, lane = row)
constexpr uint32_t T_Z1 = 0;      // Z1, later dH2 (64)
constexpr uint32_t T_Z2 = 64;     // Z2, later dH1 (64)
constexpr uint32_t T_ACC3 = 128;  // dW3 (16) / forward output (16)
constexpr uint32_t T_ACC1 = 160;  // dW1^T (16)
constexpr uint32_t T_ACC2 = 192;  // dW2^T (64)
constexpr uint32_t TMEM_COLS = 256;

constexpr long long WAIT_CYCLES = 2000000000LL;   // about one second

// byte offset of element (row r, column k) of an operand tile with K columns
__device__ __forceinline__ uint32_t kmaj(int r, int k, int K) {
    return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: no swizzle, K-major; LBO = 128 B between the two 8-column
// halves of a K=16 step, SBO = 16*K B between 8-row groups; version 1 (bit 46)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, int K) {
    const uint64_t lbo = 128u >> 4;
    const uint64_t sbo = (uint64_t)(16 * K) >> 4;
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: BF16 A and B, FP32 D, both K-major, dense
__host__ __device__ constexpr uint32_t idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(d), "l"(a), "l"(b), "r"(id), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

// C[MxN] (+)= A[M x K] B[N x K]^T, K a multiple of 16, issued as K/16 instructions
__device__ __forceinline__ void gemm(uint32_t d, uint32_t a, uint32_t b, int M, int N, int K, bool acc) {
    const uint32_t id = idesc(M, N);
    for (int s = 0; s < K / 16; ++s)
        mma_bf16(d, sdesc(a + 256u * s, K), sdesc(b + 256u * s, K), id, (acc || s > 0) ? 1u : 0u);
}

__device__ __forceinline__ void commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
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
        if (clock64() - t0 > WAIT_CYCLES) return false;
    }
}

// operands written by st.shared (and TMEM reads finished) -> visible to the MMA issuer
__device__ __forceinline__ void sync_to_mma() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 16 FP32 columns of this thread's TMEM lane; the wait sits in the same asm so the
// registers are never read before the load has landed
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint16_t bf16_bits(float x) {
    return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
__device__ __forceinline__ float bf16_round(float x) {
    return __bfloat162float(__float2bfloat16_rn(x));
}

// one row of 8*C BF16 values (already rounded, as bits) into a K-major tile
template <int C>
__device__ __forceinline__ void store_row(uint8_t *tile, int r, int K, const uint16_t *bits) {
#pragma unroll
    for (int c = 0; c < C; ++c) {
        uint4 q;
        q.x = (uint32_t)bits[8 * c + 0] | ((uint32_t)bits[8 * c + 1] << 16);
        q.y = (uint32_t)bits[8 * c + 2] | ((uint32_t)bits[8 * c + 3] << 16);
        q.z = (uint32_t)bits[8 * c + 4] | ((uint32_t)bits[8 * c + 5] << 16);
        q.w = (uint32_t)bits[8 * c + 6] | ((uint32_t)bits[8 * c + 7] << 16);
        *reinterpret_cast<uint4 *>(tile + kmaj(r, 8 * c, K)) = q;
    }
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// MODE 0: forward, writes the network output G (n x 16, FP32) for n nodes.
// MODE 1: forward recomputation + backward for the output gradient dG (n x 16), writes this
//         CTA's partial parameter gradient to part[blockIdx.x * NPARAM ...].
// X is n_pad x 16 BF16 (n_pad a multiple of 128, padded rows zero); dG has n_pad rows.
template <int MODE>
__global__ void __launch_bounds__(128, 1)
k_mlp(const float *__restrict__ params, const uint16_t *__restrict__ X, int64_t n, int64_t ntiles,
      float *__restrict__ G, const float *__restrict__ dG, float *__restrict__ part, int *__restrict__ err) {
    extern __shared__ __align__(1024) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = smem_u32(sm);
    float *s_bias = reinterpret_cast<float *>(sm + S_BIAS);
    float *s_db = reinterpret_cast<float *>(sm + S_DB);
    float *w_db = s_db + (threadIdx.x >> 5) * (NH + NH + NO);   // this warp's sums (fixed order)
    const uint32_t bar = sbase + S_BAR;
    uint32_t *s_tmem = reinterpret_cast<uint32_t *>(sm + S_TMEM);

    // weights -> BF16 operand tiles, biases -> FP32
    auto put = [&](uint32_t off, int r, int k, int K, float v) {
        *reinterpret_cast<uint16_t *>(sm + off + kmaj(r, k, K)) = bf16_bits(v);
    };
    for (int i = tid; i < NF * NH; i += 128) {          // W1[k][n], k < 16, n < 64
        const int k = i / NH, c = i % NH;
        put(S_W1T, c, k, NF, params[OFF_W1 + i]);
    }
    for (int i = tid; i < NH * NH; i += 128) {          // W2[k][n]
        const int k = i / NH, c = i % NH;
        const float v = params[OFF_W2 + i];
        put(S_W2T, c, k, NH, v);
        put(S_W2N, k, c, NH, v);
    }
    for (int i = tid; i < NH * NO; i += 128) {          // W3[k][n], k < 64, n < 16
        const int k = i / NO, c = i % NO;
        const float v = params[OFF_W3 + i];
        put(S_W3T, c, k, NH, v);
        put(S_W3N, k, c, NO, v);
    }
    for (int i = tid; i < 4 * (NH + NH + NO); i += 128) s_db[i] = 0.f;
    for (int i = tid; i < NH + NH + NO; i += 128) {
        s_bias[i] = i < NH ? params[OFF_B1 + i] : (i < 2 * NH ? params[OFF_B2 + i - NH] : params[OFF_B3 + i - 2 * NH]);
    }
    if (MODE == 1) {   // rows 64..127 of the padded M=128 operands stay zero
        for (uint32_t o = tid * 16; o < 128 * 128; o += 128 * 16) {
            *reinterpret_cast<uint4 *>(sm + S_H2T + 128 * 128 + o) = make_uint4(0, 0, 0, 0);
            *reinterpret_cast<uint4 *>(sm + S_DZ2T + 128 * 128 + o) = make_uint4(0, 0, 0, 0);
            *reinterpret_cast<uint4 *>(sm + S_DZ1T + 128 * 128 + o) = make_uint4(0, 0, 0, 0);
        }
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + S_TMEM),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    sync_to_mma();
    const uint32_t tmem = *s_tmem;
    const uint32_t lrow = tmem + ((uint32_t)(warp * 32) << 16);   // this warp's lane quarter
    const float *b1 = s_bias, *b2 = s_bias + NH, *b3 = s_bias + 2 * NH;
    const int r = tid;   // tile row = node within the tile = TMEM lane
    uint32_t phase = 0;
    bool failed = false, started = false;

    // all threads: wait for the last commit; false when the wait ran out anywhere
    auto wait_all = [&]() -> bool {
        const bool ok = bar_wait(bar, phase);
        const int all = __syncthreads_and(ok ? 1 : 0);
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (!all) return false;
        phase ^= 1u;
        return true;
    };

    for (int64_t t = blockIdx.x; t < ntiles && !failed; t += gridDim.x) {
        const int64_t node = t * TILE + r;
        // ---- features
        {
            const uint4 *src = reinterpret_cast<const uint4 *>(X + node * NF);
            const uint4 q0 = src[0], q1 = src[1];
            *reinterpret_cast<uint4 *>(sm + S_X + kmaj(r, 0, NF)) = q0;
            *reinterpret_cast<uint4 *>(sm + S_X + kmaj(r, 8, NF)) = q1;
            if (MODE == 1) {
                const uint32_t w[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
                for (int f = 0; f < NF; ++f)
                    *reinterpret_cast<uint16_t *>(sm + S_XT + kmaj(f, r, TILE)) =
                        (uint16_t)((f & 1) ? (w[f >> 1] >> 16) : (w[f >> 1] & 0xFFFFu));
            }
        }
        sync_to_mma();
        if (tid == 0) {
            gemm(tmem + T_Z1, sbase + S_X, sbase + S_W1T, 128, NH, NF, false);
            commit(bar);
        }
        if (!wait_all()) { failed = true; break; }
        // ---- layer 1 epilogue: H1 = relu(Z1 + b1)
        uint64_t m1 = 0;
        {
            uint16_t hb[NH];
#pragma unroll
            for (int c = 0; c < NH / 16; ++c) {
                float z[16];
                tmem_ld16(lrow + T_Z1 + 16 * c, z);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const float h = z[j] + b1[16 * c + j];
                    const bool pos = h > 0.f;
                    m1 |= (uint64_t)pos << (16 * c + j);
                    hb[16 * c + j] = bf16_bits(pos ? h : 0.f);
                }
            }
            store_row<NH / 8>(sm + S_H1, r, NH, hb);
            if (MODE == 1) {
#pragma unroll
                for (int j = 0; j < NH; ++j) *reinterpret_cast<uint16_t *>(sm + S_H1T + kmaj(j, r, TILE)) = hb[j];
            }
        }
        sync_to_mma();
        if (tid == 0) {
            gemm(tmem + T_Z2, sbase + S_H1, sbase + S_W2T, 128, NH, NH, false);
            commit(bar);
        }
        if (!wait_all()) { failed = true; break; }
        // ---- layer 2 epilogue: H2 = relu(Z2 + b2)
        uint64_t m2 = 0;
        {
            uint16_t hb[NH];
#pragma unroll
            for (int c = 0; c < NH / 16; ++c) {
                float z[16];
                tmem_ld16(lrow + T_Z2 + 16 * c, z);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const float h = z[j] + b2[16 * c + j];
                    const bool pos = h > 0.f;
                    m2 |= (uint64_t)pos << (16 * c + j);
                    hb[16 * c + j] = bf16_bits(pos ? h : 0.f);
                }
            }
            if (MODE == 0) {
                store_row<NH / 8>(sm + S_H2, r, NH, hb);
            } else {
#pragma unroll
                for (int j = 0; j < NH; ++j) *reinterpret_cast<uint16_t *>(sm + S_H2T + kmaj(j, r, TILE)) = hb[j];
            }
        }
        if (MODE == 0) {
            sync_to_mma();
            if (tid == 0) {
                gemm(tmem + T_ACC3, sbase + S_H2, sbase + S_W3T, 128, NO, NH, false);
                commit(bar);
            }
            if (!wait_all()) { failed = true; break; }
            float y[16];
            tmem_ld16(lrow + T_ACC3, y);
            if (node < n) {
                float4 *dst = reinterpret_cast<float4 *>(G + node * NO);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    dst[q] = make_float4(y[4 * q] + b3[4 * q], y[4 * q + 1] + b3[4 * q + 1], y[4 * q + 2] + b3[4 * q + 2],
                                         y[4 * q + 3] + b3[4 * q + 3]);
            }
            continue;
        }
        // ---- backward: dY3 = dG (BF16)
        {
            const float4 *src = reinterpret_cast<const float4 *>(dG + node * NO);
            uint16_t gb[NO];
            float gv[NO];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 v = src[q];
                gv[4 * q] = v.x; gv[4 * q + 1] = v.y; gv[4 * q + 2] = v.z; gv[4 * q + 3] = v.w;
            }
#pragma unroll
            for (int o = 0; o < NO; ++o) {
                gb[o] = bf16_bits(gv[o]);
                *reinterpret_cast<uint16_t *>(sm + S_DY3T + kmaj(o, r, TILE)) = gb[o];
                const float s = warp_sum(bf16_round(gv[o]));
                if (lane == 0) w_db[2 * NH + o] += s;
            }
            store_row<NO / 8>(sm + S_DY3, r, NO, gb);
        }
        sync_to_mma();
        if (tid == 0) {
            gemm(tmem + T_ACC3, sbase + S_H2T, sbase + S_DY3T, 128, NO, TILE, started);   // dW3
            gemm(tmem + T_Z1, sbase + S_DY3, sbase + S_W3N, 128, NH, NO, false);          // dH2
            commit(bar);
        }
        if (!wait_all()) { failed = true; break; }
        // ---- dZ2 = dH2 * relu'(Z2)
        {
            uint16_t db[NH];
#pragma unroll
            for (int c = 0; c < NH / 16; ++c) {
                float z[16];
                tmem_ld16(lrow + T_Z1 + 16 * c, z);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int jj = 16 * c + j;
                    const float d = ((m2 >> jj) & 1ull) ? z[j] : 0.f;
                    db[jj] = bf16_bits(d);
                    const float s = warp_sum(bf16_round(d));
                    if (lane == 0) w_db[NH + jj] += s;
                }
            }
            store_row<NH / 8>(sm + S_DZ2, r, NH, db);
#pragma unroll
            for (int j = 0; j < NH; ++j) *reinterpret_cast<uint16_t *>(sm + S_DZ2T + kmaj(j, r, TILE)) = db[j];
        }
        sync_to_mma();
        if (tid == 0) {
            gemm(tmem + T_ACC2, sbase + S_DZ2T, sbase + S_H1T, 128, NH, TILE, started);   // dW2^T
            gemm(tmem + T_Z2, sbase + S_DZ2, sbase + S_W2N, 128, NH, NH, false);          // dH1
            commit(bar);
        }
        if (!wait_all()) { failed = true; break; }
        // ---- dZ1 = dH1 * relu'(Z1)
        {
#pragma unroll
            for (int c = 0; c < NH / 16; ++c) {
                float z[16];
                tmem_ld16(lrow + T_Z2 + 16 * c, z);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int jj = 16 * c + j;
                    const float d = ((m1 >> jj) & 1ull) ? z[j] : 0.f;
                    *reinterpret_cast<uint16_t *>(sm + S_DZ1T + kmaj(jj, r, TILE)) = bf16_bits(d);
                    const float s = warp_sum(bf16_round(d));
                    if (lane == 0) w_db[jj] += s;
                }
            }
        }
        sync_to_mma();
        if (tid == 0) {
            gemm(tmem + T_ACC1, sbase + S_DZ1T, sbase + S_XT, 128, NF, TILE, started);    // dW1^T
            commit(bar);
        }
        if (!wait_all()) { failed = true; break; }
        started = true;
    }

    if (failed) {
        if (tid == 0) atomicExch(err, 1);
        bar_wait(bar, phase);   // bounded: let what was issued drain before the memory goes
    } else if (MODE == 1) {
        float *out = part + (int64_t)blockIdx.x * NPARAM;
        if (tid < NH) {        // TMEM lanes 0..63 hold the weight-gradient rows
            float v[16];
            if (started) tmem_ld16(lrow + T_ACC3, v); else for (int i = 0; i < 16; ++i) v[i] = 0.f;
            for (int o = 0; o < NO; ++o) out[OFF_W3 + tid * NO + o] = v[o];
            if (started) tmem_ld16(lrow + T_ACC1, v); else for (int i = 0; i < 16; ++i) v[i] = 0.f;
            for (int f = 0; f < NF; ++f) out[OFF_W1 + f * NH + tid] = v[f];
            for (int c = 0; c < NH / 16; ++c) {
                if (started) tmem_ld16(lrow + T_ACC2 + 16 * c, v); else for (int i = 0; i < 16; ++i) v[i] = 0.f;
                for (int i = 0; i < 16; ++i) out[OFF_W2 + (16 * c + i) * NH + tid] = v[i];
            }
        }   // warps 2 and 3: TMEM lanes 64..127 are the zero padding rows
        __syncthreads();
        constexpr int NB = NH + NH + NO;
        for (int i = tid; i < NB; i += 128) {
            const float v = ((s_db[i] + s_db[NB + i]) + s_db[2 * NB + i]) + s_db[3 * NB + i];
            out[i < NH ? OFF_B1 + i : (i < 2 * NH ? OFF_B2 + i - NH : OFF_B3 + i - 2 * NH)] = v;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// grad[p] = sum over CTAs of part[c][p] (fixed order)
__global__ void k_reduce_parts(const float *__restrict__ part, int nparts, float *__restrict__ grad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NPARAM) return;
    float s = 0.f;
    for (int c = 0; c < nparts; ++c) s += part[(int64_t)c * NPARAM + p];
    grad[p] = s;
}

__global__ void k_adam(float *__restrict__ w, float *__restrict__ m, float *__restrict__ v, const float *__restrict__ g,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NPARAM) return;
    const float gp = g[p];
    const float mp = b1 * m[p] + (1.f - b1) * gp;
    const float vp = b2 * v[p] + (1.f - b2) * gp * gp;
    m[p] = mp;
    v[p] = vp;
    w[p] -= lr * (mp / c1) / (sqrtf(vp / c2) + eps);
}

// ------------------------------------------------------------------ FP64 node-block kernels

// inverse of a symmetric-or-not 3x3 block (row-major) by the adjugate
__device__ __forceinline__ bool inv3(const double *a, double *o) {
    const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
    const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    if (!(fabs(det) > 0.0)) return false;
    const double id = 1.0 / det;
    o[0] = c00 * id; o[1] = (a[2] * a[7] - a[1] * a[8]) * id; o[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    o[3] = c01 * id; o[4] = (a[0] * a[8] - a[2] * a[6]) * id; o[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    o[6] = c02 * id; o[7] = (a[1] * a[6] - a[0] * a[7]) * id; o[8] = (a[0] * a[4] - a[1] * a[3]) * id;
    return true;
}

// Dinv_i = (diagonal block of A)^{-1}
__global__ void k_block_dinv(int64_t nn, const int32_t *__restrict__ diag, const double *__restrict__ A,
                             double *__restrict__ Dinv) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
        double a[9], o[9];
        const double *blk = A + (int64_t)diag[i] * 9;
        for (int k = 0; k < 9; ++k) a[k] = blk[k];
        if (!inv3(a, o))
            for (int k = 0; k < 9; ++k) o[k] = 0.0;
        for (int k = 0; k < 9; ++k) Dinv[i * 9 + k] = o[k];
    }
}

// C_i = M_i G_i Dinv_i M_i  (M_i: free-DOF mask of the node)
__global__ void k_build_C(int64_t nn, const float *__restrict__ G, const double *__restrict__ Dinv,
                          const double *__restrict__ mask, double *__restrict__ Cb) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
        const double *D = Dinv + i * 9;
        const float *g = G + i * NO;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                double s = 0.0;
                for (int k = 0; k < 3; ++k) s += (double)g[a * 3 + k] * D[k * 3 + b];
                Cb[i * 9 + a * 3 + b] = s * mask[i * 3 + a] * mask[i * 3 + b];
            }
    }
}

// y = Dinv rz (per node)
__global__ void k_block_apply(int64_t nn, const double *__restrict__ B, const double *__restrict__ x,
                              double *__restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
        const double *b = B + i * 9;
        const double x0 = x[3 * i], x1 = x[3 * i + 1], x2 = x[3 * i + 2];
        y[3 * i] = b[0] * x0 + b[1] * x1 + b[2] * x2;
        y[3 * i + 1] = b[3] * x0 + b[4] * x1 + b[5] * x2;
        y[3 * i + 2] = b[6] * x0 + b[7] * x1 + b[8] * x2;
    }
}

// v = s * (v + a q)   (q may be NULL)
__global__ void k_axpy_scale(int64_t n, double *__restrict__ v, const double *__restrict__ q, double a, double s) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = s * (v[i] + (q ? a * q[i] : 0.0));
}

// d = M (G y)   (G from the network output, FP32)
__global__ void k_apply_G(int64_t nn, const float *__restrict__ G, const double *__restrict__ mask,
                          const double *__restrict__ y, double *__restrict__ d) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
        const float *g = G + i * NO;
        const double y0 = y[3 * i], y1 = y[3 * i + 1], y2 = y[3 * i + 2];
        for (int a = 0; a < 3; ++a)
            d[3 * i + a] = mask[3 * i + a] * ((double)g[3 * a] * y0 + (double)g[3 * a + 1] * y1 + (double)g[3 * a + 2] * y2);
    }
}

// e = rz - q; per-block partial sums of |e|^2 into part[blockIdx.x]
__global__ void k_residual(int64_t n, const double *__restrict__ rz, const double *__restrict__ q,
                           double *__restrict__ e, double *__restrict__ part) {
    __shared__ double red[256];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = rz[i] - q[i];
        e[i] = v;
        s += v * v;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// e = rz - q; per-block partial sums of d . (q - 2 rz) into part[blockIdx.x] (the change of the
// energy norm of the error, |e_z - d|_A^2 - |e_z|_A^2, for rz = A e_z and q = A d)
__global__ void k_energy(int64_t n, const double *__restrict__ d, const double *__restrict__ rz,
                         const double *__restrict__ q, double *__restrict__ e, double *__restrict__ part) {
    __shared__ double red[256];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double qi = q[i], ri = rz[i];
        e[i] = ri - qi;
        s += d[i] * (qi - 2.0 * ri);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// loss[slot] += w * sum(part)   (one thread)
__global__ void k_loss_acc(const double *__restrict__ part, int nparts, double w, double *__restrict__ loss, int first) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int i = 0; i < nparts; ++i) s += part[i];
    loss[0] = (first ? 0.0 : loss[0]) + w * s;
}

// dG_i[a][b] (+)= coef * mask_ia * g_ia * y_ib
__global__ void k_grad_G(int64_t nn, double coef, const double *__restrict__ mask, const double *__restrict__ g,
                         const double *__restrict__ y, float *__restrict__ dG, int first) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
        float *o = dG + i * NO;
        for (int a = 0; a < 3; ++a) {
            const double ga = coef * mask[3 * i + a] * g[3 * i + a];
            for (int b = 0; b < 3; ++b) {
                const float v = (float)(ga * y[3 * i + b]);
                o[3 * a + b] = first ? v : o[3 * a + b] + v;
            }
        }
        if (first)
            for (int k = 9; k < NO; ++k) o[k] = 0.f;
    }
}

// ------------------------------------------------------------------ node features

// partial sums for the feature normalisation: [sum free diag, count free DOFs, sum r^2 over free
// DOFs, unused, sum c_bar] over this block's range
__global__ void k_feat_stats(int64_t nn, int64_t n_int, const int32_t *__restrict__ diag, const double *__restrict__ A,
                             const double *__restrict__ mask, const double *__restrict__ res,
                             const double *__restrict__ c_bar, double *__restrict__ part) {
    __shared__ double red[5][256];
    double s[5] = {0, 0, 0, 0, 0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
        const double *blk = A + (int64_t)diag[i] * 9;
        for (int a = 0; a < 3; ++a) {
            const double m = mask[3 * i + a];
            s[0] += m * fabs(blk[4 * a]);
            s[1] += m;
            s[2] += m * res[3 * i + a] * res[3 * i + a];
        }
    }
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n_int; p += (int64_t)gridDim.x * blockDim.x)
        s[4] += c_bar ? c_bar[p] : 0.0;
    for (int k = 0; k < 5; ++k) red[k][threadIdx.x] = s[k];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o)
            for (int k = 0; k < 5; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 5; ++k) part[blockIdx.x * 5 + k] = red[k][0];
}

// stats = [mean free diag, rms residual over free DOFs, mean c_bar]
__global__ void k_feat_stats_final(const double *__restrict__ part, int nparts, int64_t n_int,
                                   double *__restrict__ stats) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s[5] = {0, 0, 0, 0, 0};
    for (int b = 0; b < nparts; ++b)
        for (int k = 0; k < 5; ++k) s[k] += part[b * 5 + k];
    const double nfree = s[1] > 0 ? s[1] : 1.0;
    stats[0] = s[0] / nfree > 0 ? s[0] / nfree : 1.0;
    stats[1] = sqrt(s[2] / nfree) > 0 ? sqrt(s[2] / nfree) : 1.0;
    stats[2] = n_int > 0 ? s[4] / (double)n_int : 1.0;
    if (!(stats[2] > 0)) stats[2] = 1.0;
}

__device__ __forceinline__ float slog1p(double x) {
    return (float)(x >= 0 ? log1p(x) : -log1p(-x));
}

// per element: fraction of plastic integration points and mean reduced cohesion
__global__ void k_elem_stats(int64_t n_e, int nq, const uint8_t *__restrict__ branch, const double *__restrict__ c_bar,
                             float *__restrict__ eplast, double *__restrict__ ecbar) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_e; e += (int64_t)gridDim.x * blockDim.x) {
        int np_ = 0;
        double ce = 0.0;
        for (int q = 0; q < nq; ++q) {
            if (branch && branch[e * nq + q] != 0) ++np_;
            if (c_bar) ce += c_bar[e * nq + q];
        }
        eplast[e] = (float)np_ / (float)nq;
        ecbar[e] = ce / nq;
    }
}

// phi (BF16, n_pad x 16): [log10 diag / mean (3), plastic fraction, coords in [-1,1] (3),
// all-free flag, signed log1p(residual / rms) (3), log(c_bar / mean), free fraction, 0, 0, 0];
// element quantities averaged over the elements that contain the node
__global__ void k_features(int64_t nn, int64_t n_pad, const int32_t *__restrict__ n2e_ptr,
                           const int32_t *__restrict__ n2e, const int32_t *__restrict__ diag,
                           const double *__restrict__ A, const double *__restrict__ mask,
                           const float *__restrict__ coordn, const double *__restrict__ res,
                           const float *__restrict__ eplast, const double *__restrict__ ecbar, int have_c,
                           const double *__restrict__ stats, uint16_t *__restrict__ X) {
    const double dmean = stats[0], rrms = stats[1], cmean = stats[2];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_pad; i += (int64_t)gridDim.x * blockDim.x) {
        float f[NF];
        for (int k = 0; k < NF; ++k) f[k] = 0.f;
        if (i < nn) {
            const double *blk = A + (int64_t)diag[i] * 9;
            double mfree = 0.0;
            for (int a = 0; a < 3; ++a) {
                const double dv = fabs(blk[4 * a]);
                f[a] = (float)log10((dv > 1e-300 ? dv : 1e-300) / dmean);
                f[8 + a] = slog1p(res[3 * i + a] / rrms);
                mfree += mask[3 * i + a];
            }
            double plast = 0.0, cs = 0.0;
            const int32_t k0 = n2e_ptr[i], k1 = n2e_ptr[i + 1];
            for (int32_t k = k0; k < k1; ++k) {
                plast += eplast[n2e[k]];
                cs += ecbar[n2e[k]];
            }
            if (k1 > k0) {
                f[3] = (float)(plast / (k1 - k0));
                const double cn = cs / (k1 - k0);
                f[11] = have_c ? (float)log((cn > 1e-300 ? cn : 1e-300) / cmean) : 0.f;
            }
            f[4] = coordn[3 * i];
            f[5] = coordn[3 * i + 1];
            f[6] = coordn[3 * i + 2];
            f[7] = mfree == 3.0 ? 1.f : 0.f;
            f[12] = (float)(mfree / 3.0);
        }
        uint32_t w[8];
        for (int k = 0; k < 8; ++k) w[k] = (uint32_t)bf16_bits(f[2 * k]) | ((uint32_t)bf16_bits(f[2 * k + 1]) << 16);
        reinterpret_cast<uint4 *>(X + i * NF)[0] = make_uint4(w[0], w[1], w[2], w[3]);
        reinterpret_cast<uint4 *>(X + i * NF)[1] = make_uint4(w[4], w[5], w[6], w[7]);
    }
}

int mlp_launch(int mode, const float *params, const uint16_t *X, int64_t n, float *G, const float *dG, float *part,
               int nparts, int *err, cudaStream_t st) {
    const int64_t ntiles = (n + TILE - 1) / TILE;
    static int attr_done[2] = {0, 0};
    if (!attr_done[mode]) {
        if (mode == 0)
            SG_CUDA(cudaFuncSetAttribute(k_mlp<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES));
        else
            SG_CUDA(cudaFuncSetAttribute(k_mlp<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES));
        attr_done[mode] = 1;
    }
    count_launch();
    if (mode == 0)
        k_mlp<0><<<nparts, 128, SMEM_BYTES, st>>>(params, X, n, ntiles, G, nullptr, nullptr, err);
    else
        k_mlp<1><<<nparts, 128, SMEM_BYTES, st>>>(params, X, n, ntiles, nullptr, dG, part, err);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

int mlp_grid(int64_t n) {
    const int64_t ntiles = (n + TILE - 1) / TILE;
    const int64_t g = ntiles < sm_count() ? ntiles : sm_count();
    return (int)(g < 1 ? 1 : g);
}

}  // namespace lc
}  // namespace sg

using namespace sg;
using namespace sg::lc;

// ------------------------------------------------------------------ stateless network entry points

// G (n x 16 FP32) = MLP(params; X (n_pad x 16 BF16 bits)), device pointers
extern "C" int sg_mlp_forward_dev(const float *params, const uint16_t *X, int64_t n, float *G, int *err, void *stream) {
    SG_CHECK_ARG(params && X && G && err && n > 0, "bad argument");
    return mlp_launch(0, params, X, n, G, nullptr, nullptr, mlp_grid(n), err, as_stream(stream));
}

// grad (NPARAM FP32) = d/dparams sum_i <dG_i, MLP(params; X_i)>; part: scratch of
// sg_mlp_part_size(n) floats; X and dG have n_pad = 128 * ceil(n/128) rows (padding rows zero)
extern "C" int64_t sg_mlp_part_size(int64_t n) { return (int64_t)mlp_grid(n) * NPARAM; }

extern "C" int sg_mlp_backward_dev(const float *params, const uint16_t *X, const float *dG, int64_t n, float *grad,
                                   float *part, int *err, void *stream) {
    SG_CHECK_ARG(params && X && dG && grad && part && err && n > 0, "bad argument");
    const cudaStream_t st = as_stream(stream);
    const int g = mlp_grid(n);
    int rc = mlp_launch(1, params, X, n, nullptr, dG, part, g, err, st);
    if (rc) return rc;
    k_reduce_parts<<<grid_for(NPARAM, 256), 256, 0, st>>>(part, g, grad);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

// ------------------------------------------------------------------ the learned correction

struct sg_learned {
    const sg_mesh *mesh = nullptr;
    int64_t nn = 0, n_pad = 0, nd = 0;
    int max_vec = 0, n_vec[2] = {0, 0};
    float *params = nullptr, *adam_m = nullptr, *adam_v = nullptr, *grad = nullptr, *part = nullptr;
    float *G = nullptr, *dG = nullptr, *coordn = nullptr, *eplast = nullptr;
    double *ecbar = nullptr;
    uint16_t *X = nullptr;
    int32_t *n2e_ptr = nullptr, *n2e = nullptr;
    double *Dinv = nullptr, *C = nullptr, *stats = nullptr, *spart = nullptr;
    double *rz[2] = {nullptr, nullptr}, *y[2] = {nullptr, nullptr};   // [slot][vec * nd]
    double *nrm[2] = {nullptr, nullptr};                               // host copies of |rz|^2
    double *nrmE[2] = {nullptr, nullptr};                              // host copies of rz' Dinv rz
    int loss_kind = 0;                                                 // 0 residual, 1 energy
    double *v = nullptr, *z = nullptr, *d = nullptr, *q = nullptr, *e = nullptr, *g = nullptr;
    double *loss = nullptr, *lpart = nullptr;
    int *err = nullptr;
    int adam_t = 0;
    int have_features = 0;
};

static int lfree(sg_learned *h) {
    void *ps[] = {h->params, h->adam_m, h->adam_v, h->grad, h->part, h->G, h->dG, h->coordn, h->eplast, h->ecbar, h->X, h->n2e_ptr, h->n2e,
                  h->Dinv, h->C, h->stats, h->spart, h->rz[0], h->rz[1], h->y[0], h->y[1], h->v, h->z, h->d, h->q,
                  h->e, h->g, h->loss, h->lpart, h->err};
    for (void *p : ps)
        if (p) cudaFree(p);
    delete[] h->nrm[0];
    delete[] h->nrm[1];
    delete[] h->nrmE[0];
    delete[] h->nrmE[1];
    delete h;
    return SG_OK;
}

template <typename T>
static int zalloc(T **p, size_t n) {
    *p = nullptr;
    SG_CUDA(sg::device_alloc((void **)p, (n ? n : 1) * sizeof(T)));
    SG_CUDA(cudaMemset(*p, 0, (n ? n : 1) * sizeof(T)));
    return SG_OK;
}

// Network initialisation: He-uniform first two layers (seeded), last layer zero, so the
// untrained correction is exactly zero.
static void init_params(std::vector<float> &P, uint64_t seed) {
    P.assign(NPARAM, 0.f);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<float> u(-1.f, 1.f);
    const float a1 = std::sqrt(6.f / NF), a2 = std::sqrt(6.f / NH);
    for (int i = 0; i < NF * NH; ++i) P[OFF_W1 + i] = a1 * u(rng);
    for (int i = 0; i < NH * NH; ++i) P[OFF_W2 + i] = a2 * u(rng);
    for (int i = 0; i < NH; ++i) P[OFF_B1 + i] = 0.01f;
    for (int i = 0; i < NH; ++i) P[OFF_B2 + i] = 0.01f;
}

extern "C" int sg_learned_create(const sg_mesh *mesh, const double *coord, int32_t max_vectors, uint64_t seed,
                                 sg_learned **out) {
    SG_CHECK_ARG(out, "null output handle");
    *out = nullptr;
    SG_CHECK_ARG(mesh && coord && max_vectors > 0, "bad argument");
    SG_CHECK_ARG(mesh->dim == 3, "the learned correction is defined for 3D meshes (3 x 3 node blocks)");
    sg_learned *h = new (std::nothrow) sg_learned();
    if (!h) return set_error(SG_ERR_NOMEM, "host allocation");
    h->mesh = mesh;
    h->nn = mesh->n_n;
    h->n_pad = (h->nn + TILE - 1) / TILE * TILE;
    h->nd = 3 * h->nn;
    h->max_vec = max_vectors;
    h->nrm[0] = new double[max_vectors]();
    h->nrm[1] = new double[max_vectors]();
    h->nrmE[0] = new double[max_vectors]();
    h->nrmE[1] = new double[max_vectors]();
    int rc = SG_OK;
    const int gparts = mlp_grid(h->nn);
#define LA(p, n) if (!rc) rc = zalloc(&(p), (size_t)(n))
    LA(h->params, NPARAM); LA(h->adam_m, NPARAM); LA(h->adam_v, NPARAM); LA(h->grad, NPARAM);
    LA(h->part, (size_t)gparts * NPARAM);
    LA(h->G, h->n_pad * NO); LA(h->dG, h->n_pad * NO); LA(h->X, h->n_pad * NF); LA(h->coordn, h->nd); LA(h->eplast, mesh->n_e); LA(h->ecbar, mesh->n_e);
    LA(h->Dinv, h->nn * 9); LA(h->C, h->nn * 9); LA(h->stats, 4); LA(h->spart, 5 * 4096);
    for (int s = 0; s < 2; ++s) { LA(h->rz[s], (size_t)max_vectors * h->nd); LA(h->y[s], (size_t)max_vectors * h->nd); }
    LA(h->v, h->nd); LA(h->z, h->nd); LA(h->d, h->nd); LA(h->q, h->nd); LA(h->e, h->nd); LA(h->g, h->nd);
    LA(h->loss, 4); LA(h->lpart, 4096); LA(h->err, 1);
#undef LA
    if (rc) { lfree(h); return rc; }
    // coordinates scaled to [-1, 1] per axis; node -> element incidence (CSR)
    std::vector<float> cn(h->nd);
    for (int a = 0; a < 3; ++a) {
        double lo = 1e300, hi = -1e300;
        for (int64_t i = 0; i < h->nn; ++i) { lo = std::min(lo, coord[a + 3 * i]); hi = std::max(hi, coord[a + 3 * i]); }
        const double span = hi > lo ? hi - lo : 1.0;
        for (int64_t i = 0; i < h->nn; ++i) cn[3 * i + a] = (float)(2.0 * (coord[a + 3 * i] - lo) / span - 1.0);
    }
    std::vector<int32_t> ptr(h->nn + 1, 0), inc;
    for (int64_t e = 0; e < mesh->n_e; ++e)
        for (int k = 0; k < mesh->np; ++k) ptr[mesh->elem[e * mesh->np + k] + 1]++;
    for (int64_t i = 0; i < h->nn; ++i) ptr[i + 1] += ptr[i];
    inc.resize(ptr[h->nn]);
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int64_t e = 0; e < mesh->n_e; ++e)
        for (int k = 0; k < mesh->np; ++k) inc[fill[mesh->elem[e * mesh->np + k]]++] = (int32_t)e;
    std::vector<float> P;
    init_params(P, seed);
    if (!rc) rc = zalloc(&h->n2e_ptr, ptr.size());
    if (!rc) rc = zalloc(&h->n2e, inc.size());
    if (rc) { lfree(h); return rc; }
    cudaError_t ce = cudaMemcpy(h->coordn, cn.data(), sizeof(float) * cn.size(), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemcpy(h->n2e_ptr, ptr.data(), sizeof(int32_t) * ptr.size(), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess && !inc.empty())
        ce = cudaMemcpy(h->n2e, inc.data(), sizeof(int32_t) * inc.size(), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemcpy(h->params, P.data(), sizeof(float) * NPARAM, cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) { lfree(h); return cuda_error(ce, "learned correction set-up copies"); }
    *out = h;
    return SG_OK;
}

extern "C" int sg_learned_destroy(sg_learned *h) {
    if (!h) return SG_OK;
    return lfree(h);
}

// host <-> device parameter vector (NPARAM floats); set resets the optimiser state
extern "C" int sg_learned_params(sg_learned *h, float *host, int32_t set) {
    SG_CHECK_ARG(h && host, "bad argument");
    if (set) {
        SG_CUDA(cudaMemcpy(h->params, host, sizeof(float) * NPARAM, cudaMemcpyHostToDevice));
        SG_CUDA(cudaMemset(h->adam_m, 0, sizeof(float) * NPARAM));
        SG_CUDA(cudaMemset(h->adam_v, 0, sizeof(float) * NPARAM));
        h->adam_t = 0;
    } else {
        SG_CUDA(cudaMemcpy(host, h->params, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
    }
    return SG_OK;
}

static int check_err(sg_learned *h) {
    int e = 0;
    SG_CUDA(cudaMemcpy(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        cudaMemset(h->err, 0, sizeof(int));
        return set_error(SG_ERR_STATE, "tensor-core network kernel: an MMA completion wait ran out");
    }
    return SG_OK;
}

// Node features from the matrix A (device values on the mesh pattern), the Newton residual
// res (device, dim*n_n), the per-point branch ids and reduced cohesion (device, may be NULL),
// then Dinv = diagonal-block inverses of A.
extern "C" int sg_learned_features(sg_learned *h, const double *A_vals, const double *res, const uint8_t *branch,
                                   const double *c_bar, void *stream) {
    SG_CHECK_ARG(h && A_vals && res, "bad argument");
    const cudaStream_t st = as_stream(stream);
    const sg_mesh *m = h->mesh;
    const int nb = 256;
    const unsigned gs = grid_for(std::max<int64_t>(h->nn, m->n_int), 256, 8);
    SG_CHECK_ARG(gs <= 4096, "grid too large");
    k_feat_stats<<<gs, 256, 0, st>>>(h->nn, c_bar ? m->n_int : 0, m->bsr.d_diag, A_vals, m->d_mask, res, c_bar, h->spart);
    count_launch();
    k_feat_stats_final<<<1, 32, 0, st>>>(h->spart, (int)gs, c_bar ? m->n_int : 0, h->stats);
    k_elem_stats<<<grid_for(m->n_e, nb), nb, 0, st>>>(m->n_e, m->nq, branch, c_bar, h->eplast, h->ecbar);
    k_features<<<grid_for(h->n_pad, nb), nb, 0, st>>>(h->nn, h->n_pad, h->n2e_ptr, h->n2e, m->bsr.d_diag, A_vals,
                                                    m->d_mask, h->coordn, res, h->eplast, h->ecbar, c_bar ? 1 : 0,
                                                    h->stats, h->X);
    k_block_dinv<<<grid_for(h->nn, nb), nb, 0, st>>>(h->nn, m->bsr.d_diag, A_vals, h->Dinv);
    SG_CUDA(cudaGetLastError());
    h->have_features = 1;
    return SG_OK;
}

// C = M G Dinv M from the current parameters and features; optionally handed to the AMG
// instance (amg may be NULL).  C_out (device, n_n*9) may be NULL.
extern "C" int sg_learned_correction(sg_learned *h, sg_amg *amg, double *C_out, void *stream) {
    SG_CHECK_ARG(h, "bad argument");
    if (!h->have_features) return set_error(SG_ERR_STATE, "sg_learned_features must be called first");
    const cudaStream_t st = as_stream(stream);
    int rc = mlp_launch(0, h->params, h->X, h->nn, h->G, nullptr, nullptr, mlp_grid(h->nn), h->err, st);
    if (rc) return rc;
    k_build_C<<<grid_for(h->nn, 256), 256, 0, st>>>(h->nn, h->G, h->Dinv, h->mesh->d_mask, h->C);
    SG_CUDA(cudaGetLastError());
    if ((rc = check_err(h))) return rc;
    if (C_out) SG_CUDA(cudaMemcpyAsync(C_out, h->C, sizeof(double) * h->nn * 9, cudaMemcpyDeviceToDevice, st));
    if (amg) return sg_amg_set_correction(amg, h->C, stream);
    return SG_OK;
}

// Harvest `count` training vectors into slot (0 training, 1 held out) from the right-hand
// side b: v_0 = b/|b|; z = V(v) with the plain V-cycle; rz = v - A z; stored (rz, Dinv rz);
// the next v is the minimal-residual update v - a A z (normalised), the residual sequence a
// preconditioned Richardson/GMRES(1) iteration on A x = b produces.  sg_learned_features
// must have been called for A (Dinv).
extern "C" int sg_learned_collect(sg_learned *h, sg_amg *amg, const sg_bsr *A, const double *A_vals, const double *b,
                                  int32_t count, int32_t slot, int32_t append, void *stream) {
    SG_CHECK_ARG(h && amg && A && A_vals && b && count > 0 && (slot == 0 || slot == 1), "bad argument");
    if (!h->have_features) return set_error(SG_ERR_STATE, "sg_learned_features must be called first");
    const int base = append ? h->n_vec[slot] : 0;
    SG_CHECK_ARG(base + count <= h->max_vec, "more vectors than the handle holds");
    const cudaStream_t st = as_stream(stream);
    const int64_t nd = h->nd;
    int rc = sg_amg_set_correction(amg, nullptr, stream);   // plain V-cycle while collecting
    if (rc) return rc;
    SG_CUDA(cudaMemcpyAsync(h->v, b, sizeof(double) * nd, cudaMemcpyDeviceToDevice, st));
    for (int k = 0; k < count; ++k) {
        double vv = 0.0, vq = 0.0, qq = 0.0, rr = 0.0;
        if ((rc = sg_dot_dev(nd, h->v, h->v, &vv, stream))) return rc;
        if (!(vv > 0.0) || !std::isfinite(vv)) return set_error(SG_ERR_NUMERIC, "zero or non-finite vector while collecting");
        k_axpy_scale<<<grid_for(nd, 256), 256, 0, st>>>(nd, h->v, nullptr, 0.0, 1.0 / std::sqrt(vv));
        if ((rc = sg_amg_apply(amg, h->v, h->z, stream))) return rc;
        if ((rc = sg_bsr_spmv_dev(A, A_vals, h->z, h->q, stream))) return rc;   // q = A z
        double *rzk = h->rz[slot] + (int64_t)(base + k) * nd, *yk = h->y[slot] + (int64_t)(base + k) * nd;
        k_residual<<<grid_for(nd, 256), 256, 0, st>>>(nd, h->v, h->q, rzk, h->lpart);
        k_block_apply<<<grid_for(h->nn, 256), 256, 0, st>>>(h->nn, h->Dinv, rzk, yk);
        SG_CUDA(cudaGetLastError());
        if ((rc = sg_dot_dev(nd, h->v, h->q, &vq, stream))) return rc;
        if ((rc = sg_dot_dev(nd, h->q, h->q, &qq, stream))) return rc;
        if ((rc = sg_dot_dev(nd, rzk, rzk, &rr, stream))) return rc;
        h->nrm[slot][base + k] = rr;
        double ry = 0.0;
        if ((rc = sg_dot_dev(nd, rzk, yk, &ry, stream))) return rc;
        h->nrmE[slot][base + k] = ry;
        // next v = v - a q, a = (v.q)/(q.q): the residual of one minimal-residual step
        k_axpy_scale<<<grid_for(nd, 256), 256, 0, st>>>(nd, h->v, h->q, qq > 0 ? -vq / qq : 0.0, 1.0);
        SG_CUDA(cudaGetLastError());
    }
    SG_CUDA(cudaStreamSynchronize(st));
    h->n_vec[slot] = base + count;
    return SG_OK;
}

// training objective over slot's vectors with the current network (sg_learned_set_loss);
// when want_grad also dG (dL/dG), left in the handle.
static int loss_pass(sg_learned *h, const sg_bsr *A, const double *A_vals, int slot, bool want_grad, cudaStream_t st) {
    const int S = h->n_vec[slot];
    if (S <= 0) return set_error(SG_ERR_STATE, "no vectors collected in this slot");
    const int64_t nd = h->nd, nn = h->nn;
    int rc = mlp_launch(0, h->params, h->X, nn, h->G, nullptr, nullptr, mlp_grid(nn), h->err, st);
    if (rc) return rc;
    const unsigned gr = grid_for(nd, 256);
    for (int s = 0; s < S; ++s) {
        const double *rzs = h->rz[slot] + (int64_t)s * nd, *ys = h->y[slot] + (int64_t)s * nd;
        const bool energy = h->loss_kind == 1;
        const double nr = energy ? h->nrmE[slot][s] : h->nrm[slot][s];
        const double w = 1.0 / (S * (nr > 0 ? nr : 1.0));
        k_apply_G<<<grid_for(nn, 256), 256, 0, st>>>(nn, h->G, h->mesh->d_mask, ys, h->d);
        if ((rc = sg_bsr_spmv_dev(A, A_vals, h->d, h->q, st))) return rc;
        if (energy)
            k_energy<<<gr, 256, 0, st>>>(nd, h->d, rzs, h->q, h->e, h->lpart);
        else
            k_residual<<<gr, 256, 0, st>>>(nd, rzs, h->q, h->e, h->lpart);
        count_launch();
        k_loss_acc<<<1, 32, 0, st>>>(h->lpart, (int)gr, w, h->loss, s == 0);
        if (want_grad) {
            // residual loss: dL/dd = -2 w A e;  energy loss: dL/dd = 2 w (A d - rz) = -2 w e
            const double *g = h->e;
            if (!energy) {
                if ((rc = sg_bsr_spmv_dev(A, A_vals, h->e, h->g, st))) return rc;
                g = h->g;
            }
            k_grad_G<<<grid_for(nn, 256), 256, 0, st>>>(nn, -2.0 * w, h->mesh->d_mask, g, ys, h->dG, s == 0);
        }
        SG_CUDA(cudaGetLastError());
    }
    return SG_OK;
}

// training objective: 0 (default) the mean relative residual |rz - A d|^2 / |rz|^2, 1 the
// mean change of the error's energy norm (|e_z - d|_A^2 - |e_z|_A^2) / (rz' D^{-1} rz)
extern "C" int sg_learned_set_loss(sg_learned *h, int32_t kind) {
    SG_CHECK_ARG(h && (kind == 0 || kind == 1), "bad argument");
    h->loss_kind = kind;
    return SG_OK;
}

extern "C" int sg_learned_loss(sg_learned *h, const sg_bsr *A, const double *A_vals, int32_t slot, double *loss,
                               void *stream) {
    SG_CHECK_ARG(h && A && A_vals && loss && (slot == 0 || slot == 1), "bad argument");
    if (!h->have_features) return set_error(SG_ERR_STATE, "sg_learned_features must be called first");
    const cudaStream_t st = as_stream(stream);
    int rc = loss_pass(h, A, A_vals, slot, false, st);
    if (rc) return rc;
    SG_CUDA(cudaMemcpyAsync(loss, h->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    return check_err(h);
}

// dL/dparams for slot's vectors at the current parameters (host array of NPARAM floats), and
// the loss; for gradient checks
extern "C" int sg_learned_gradient(sg_learned *h, const sg_bsr *A, const double *A_vals, int32_t slot, float *grad,
                                   double *loss, void *stream) {
    SG_CHECK_ARG(h && A && A_vals && grad && (slot == 0 || slot == 1), "bad argument");
    if (!h->have_features) return set_error(SG_ERR_STATE, "sg_learned_features must be called first");
    const cudaStream_t st = as_stream(stream);
    int rc = loss_pass(h, A, A_vals, slot, true, st);
    if (!rc) rc = sg_mlp_backward_dev(h->params, h->X, h->dG, h->nn, h->grad, h->part, h->err, stream);
    if (rc) return rc;
    SG_CUDA(cudaMemcpyAsync(grad, h->grad, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, st));
    if (loss) SG_CUDA(cudaMemcpyAsync(loss, h->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    return check_err(h);
}

// `steps` Adam steps (full batch over slot 0) with learning rate lr; loss_hist (host, may be
// NULL) receives the training loss before each step.
extern "C" int sg_learned_train(sg_learned *h, const sg_bsr *A, const double *A_vals, int32_t steps, double lr,
                                double *loss_hist, void *stream) {
    SG_CHECK_ARG(h && A && A_vals && steps >= 0, "bad argument");
    if (!h->have_features) return set_error(SG_ERR_STATE, "sg_learned_features must be called first");
    const cudaStream_t st = as_stream(stream);
    double *dl = nullptr;
    if (loss_hist && steps > 0) SG_CUDA(sg::device_alloc(&dl, sizeof(double) * steps));
    int rc = SG_OK;
    const float b1 = 0.9f, b2 = 0.999f;
    for (int k = 0; k < steps && !rc; ++k) {
        rc = loss_pass(h, A, A_vals, 0, true, st);
        if (!rc && dl) {
            cudaError_t ce = cudaMemcpyAsync(dl + k, h->loss, sizeof(double), cudaMemcpyDeviceToDevice, st);
            if (ce != cudaSuccess) rc = cuda_error(ce, "loss copy");
        }
        if (!rc) rc = sg_mlp_backward_dev(h->params, h->X, h->dG, h->nn, h->grad, h->part, h->err, stream);
        if (!rc) {
            h->adam_t++;
            const float c1 = 1.f - std::pow(b1, (float)h->adam_t), c2 = 1.f - std::pow(b2, (float)h->adam_t);
            k_adam<<<grid_for(NPARAM, 256), 256, 0, st>>>(h->params, h->adam_m, h->adam_v, h->grad, (float)lr, b1, b2,
                                                         1e-8f, c1, c2);
            cudaError_t ce = cudaGetLastError();
            if (ce != cudaSuccess) rc = cuda_error(ce, "adam");
        }
    }
    if (!rc && dl) {
        cudaError_t ce = cudaMemcpyAsync(loss_hist, dl, sizeof(double) * steps, cudaMemcpyDeviceToHost, st);
        if (ce != cudaSuccess) rc = cuda_error(ce, "loss history copy");
    }
    if (!rc) {
        cudaError_t ce = cudaStreamSynchronize(st);
        if (ce != cudaSuccess) rc = cuda_error(ce, "train sync");
    }
    if (dl) cudaFree(dl);
    if (!rc) rc = check_err(h);
    return rc;
}

// host copy of internal state, for checks: what 0 features (n_pad x 16 BF16 bits), 1 the last
// network output G (n_pad x 16 FP32), 2 Dinv (n_n x 9 FP64), 3 / 4 residual vector `index` of
// slot 0 / 1 (dim*n_n FP64), 5 the correction C (n_n x 9 FP64)
extern "C" int sg_learned_export(const sg_learned *h, int32_t what, int32_t index, void *host) {
    SG_CHECK_ARG(h && host && what >= 0 && what <= 5, "bad argument");
    const void *src = nullptr;
    size_t bytes = 0;
    switch (what) {
        case 0: src = h->X; bytes = sizeof(uint16_t) * h->n_pad * NF; break;
        case 1: src = h->G; bytes = sizeof(float) * h->n_pad * NO; break;
        case 2: src = h->Dinv; bytes = sizeof(double) * h->nn * 9; break;
        case 3:
        case 4: {
            const int slot = what - 3;
            SG_CHECK_ARG(index >= 0 && index < h->n_vec[slot], "vector index out of range");
            src = h->rz[slot] + (int64_t)index * h->nd;
            bytes = sizeof(double) * h->nd;
            break;
        }
        default: src = h->C; bytes = sizeof(double) * h->nn * 9; break;
    }
    SG_CUDA(cudaDeviceSynchronize());
    SG_CUDA(cudaMemcpy(host, src, bytes, cudaMemcpyDeviceToHost));
    return SG_OK;
}

extern "C" int sg_learned_info(const sg_learned *h, int64_t *info) {
    SG_CHECK_ARG(h && info, "bad argument");
    info[0] = NPARAM;
    info[1] = h->n_vec[0];
    info[2] = h->n_vec[1];
    info[3] = h->n_pad;
    info[4] = h->adam_t;
    return SG_OK;
}
