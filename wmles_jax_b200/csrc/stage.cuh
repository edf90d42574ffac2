// Launch interface of the fused stage kernel (stage.cu).
#pragma once
#include "wm_internal.cuh"

namespace wm {

struct StageOpts {
    int precision;   // WM_PREC_*
    int scheme;      // WM_SCHEME_*
    int kep_order;   // 2 or 4
    int limiter;     // WM_LIMITER_*
    int sgs;         // WM_SGS_*
    int tile;        // tile shape id
};

cudaError_t launch_stage(const StageArgs& A, const StageOpts& o, cudaStream_t s);
void tile_shape(int tile, int* tj, int* tk);
int stage_ctas_per_sm(const StageOpts& o);

}  // namespace wm
