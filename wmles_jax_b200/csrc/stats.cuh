// Plane statistics kernel (stats.cu).
#pragma once
#include "wm_internal.cuh"

namespace wm {

constexpr int PS_NQ = 12;        // rho, u, v, w, uu, vv, ww, uv, uw, vw, T, p
constexpr int PS_CHUNKS = 8;     // i-chunks per plane (CTAs per plane)

struct PlaneStatsArgs {
    const BlockDev* block;       // device descriptor of the block
    const double* q;             // its state
    double gm1, Rg;
    int nchunks;
    double* part;                // scratch: PS_NQ x nj x nchunks partial sums
    double* sum;                 // accumulator: PS_NQ x nj, plane means added
    unsigned int* counter;       // last-CTA-done counter (reset by the last CTA)
};

cudaError_t launch_plane_stats(const PlaneStatsArgs& A, int nj, cudaStream_t s);

}  // namespace wm
