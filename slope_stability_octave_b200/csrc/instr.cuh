// Sampled CUDA-event timing of selected kernel kinds (see instr.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sg {

enum InstrKind {
    IK_SPMV3_F64 = 0,    // node-block (3x3 or 2x2) SpMV, FP64 values
    IK_SPMV3_F32 = 1,    // the same, FP32 values (mixed-precision V-cycle)
    IK_CONST_SDS = 2,    // return mapping with tangent
    IK_CONST_S = 3,      // return mapping, stress only
    IK_ASSEMBLY = 4,     // tangent assembly into the block pattern
    IK_AMG_UPDATE = 5,   // AMG numeric set-up for new level-0 values (all levels)
    IK_AMG_APPLY = 6,    // one AMG V-cycle (with conversions and the optional correction)
    IK_SPMV3_F16 = 7,    // level-0 SpMV of the FP32 V-cycle on the FP16 copy of the matrix
    IK_SPMV3_F64_AORTH = 8,  // FP64 node-block SpMVs of the deflation-basis A-orthogonalisation
                             // (these may run beside an AMG update on another stream)
    IK_RESIDUAL = 9,     // fused stress-only residual F = B'(w S(B U))
    IK_SPMM_AORTH = 10,  // FP64 node-block SpMM (several vectors per pass) of the A-orthogonalisation
    IK_AORTH = 11,       // the whole A-orthogonalisation of a deflation basis (units: basis columns)
    IK_COUNT = 12
};

// Units of work done by launches of a kind (e.g. vectors multiplied by one SpMM launch), added
// while timing is enabled and read by sg_instr_units.
void instr_units(int kind, int64_t units);

// While an InstrRedirect lives on a thread, launches of kind `from` on that thread are
// counted and timed as kind `to`.
struct InstrRedirect {
    int saved_from, saved_to;
    InstrRedirect(int from, int to);
    ~InstrRedirect();
};

struct InstrToken {
    int kind = -1;
    cudaEvent_t a = nullptr, b = nullptr;
};

// While an InstrSuspend lives on a thread, nothing is timed or counted (stream capture into a
// CUDA graph, whose loop bodies cannot hold event records).
struct InstrSuspend {
    bool saved;
    InstrSuspend();
    ~InstrSuspend();
};

InstrToken instr_begin(int kind, cudaStream_t st);
void instr_end(const InstrToken &t, cudaStream_t st);

}  // namespace sg
