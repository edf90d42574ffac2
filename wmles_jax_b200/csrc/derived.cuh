// Derived output fields kernel (derived.cu).
#pragma once
#include "wm_internal.cuh"

namespace wm {

struct DerivedArgs {
    const BlockDev* block;       // device descriptor of the block
    const CaseDev* cs;           // its case's constants
    int sgs;                     // WM_SGS_* of the case
    const double* q;             // state with the first ghost layer filled
    double* out;                 // WM_NDERIVED x ni x nj x nk (interior only)
};

cudaError_t launch_derived(const DerivedArgs& A, long long cells, cudaStream_t s);

}  // namespace wm
