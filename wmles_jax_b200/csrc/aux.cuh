// Argument blocks and launchers of the surface and reduction kernels.
#pragma once
#include "wm_internal.cuh"

namespace wm {

struct GhostArgs {
    const GhostSeg* segs;     // device table, one segment per case
    int nseg;
    int total;                // entries over all segments
    double* stash;            // non-null: two-phase gather/scatter (5 x total)
    double* q[WM_MAX_BLOCKS];
    long long ncell[WM_MAX_BLOCKS];
};

struct WallArgs {
    const BlockDev* blocks;
    const CaseDev* cases;
    WallDev* walls;
    int nwalls;
    int max_faces;
    const double* q[WM_MAX_BLOCKS];
};

constexpr int DT_NT = 256;   // threads (= interior cells) per CTA of the CFL / constraint pass

struct DtArgs {
    const BlockDev* blocks;
    const CaseDev* cases;
    int nblocks;
    int ncta;                              // chunks of DT_NT interior cells, numbered block by block
    int cta_start[WM_MAX_BLOCKS + 1];      // chunks of block b: [cta_start[b], cta_start[b+1])
    int ncases;
    int case_block_start[MAX_CASES + 1];   // blocks of case c: [start[c], start[c+1])
    double* q[WM_MAX_BLOCKS];      // state (modified in place when the constraint is applied)
    const double* cmf_delta;       // per case: constant-mass-flux shift from stage 3 (null: none)
    int want_dt;                   // 0: constraint only
    int met32;                     // read the float metric copy (mixed form)
    unsigned long long* dt_key;    // per case: running minimum as an order-preserving key
                                   // (DT_KEY_EMPTY between calls: reset by the last CTA)
    unsigned int* counter;         // last-CTA-done counter (reset by the last CTA)
    double* dt_out[MAX_CASES];     // per case: time step
};

// key of DBL_MAX, the value of an empty minimum (the reset value of DtArgs::dt_key)
constexpr unsigned long long DT_KEY_EMPTY = 0xFFEFFFFFFFFFFFFFull;

struct SpongeArgs {
    const BlockDev* blocks;
    const CaseDev* cases;
    int nblocks;
    const double* q[WM_MAX_BLOCKS];
    double* mean[WM_MAX_BLOCKS];   // 5 x Ni x Nj
};

struct InflowArgs {
    const BlockDev* block;
    const double* modes;     // 3 x 4 x n_modes
    const double* table;     // n_tab x 7
    int n_modes, n_tab;
    double U_inf, L, rho_inf, p_inf, gm1;
    double time0, time_dt;   // time = time0 + time_dt * (*dt)
    const double* dt;
    double* raw;             // IN_PARTS x (ng * Nj) x 3 x Nk partial mode sums (scratch)
    double* out;             // 5 x (ng * Nj * Nk)
};

// partial mode sums per (component, cell) of the synthetic inflow (contiguous mode ranges)
constexpr int IN_PARTS = 4;
// kernel launches of one inflow fill
constexpr int IN_LAUNCHES = 2;

// before each stage kernel: ghost gather (single phase), wall model and sponge means in one
// launch; the CTA counts are filled in by the launcher (an empty part has none)
struct SurfaceArgs {
    GhostArgs G;
    WallArgs W;
    SpongeArgs S;          // nblocks = 0: no sponge
    int g_ctas, w_per, w_ctas, s_per, s_ctas;
};

__device__ __forceinline__ long long cell_index(const BlockDev& B, int axis, int c, int a, int b) {
    // cell at position c along `axis`, (a, b) on the other two axes in increasing order
    const int Nj = B.N[1], Nk = B.N[2];
    if (axis == 0) return ((long long)c * Nj + a) * Nk + b;
    if (axis == 1) return ((long long)a * Nj + c) * Nk + b;
    return ((long long)a * Nj + b) * Nk + c;
}

// Sutherland viscosity in FP64 (wmles/gas.py:39-41)
__device__ __forceinline__ double sutherland_d(double T, const CaseDev& C) {
    const double x = T * C.inv_Tref;
    return C.mu_ref * (x * sqrt(x)) * C.TrefS / (T + C.S_suth);
}

cudaError_t launch_ghost(const GhostArgs& G, cudaStream_t s);
cudaError_t launch_surface(SurfaceArgs& A, int max_sponge_rows, cudaStream_t s);
cudaError_t launch_wall(const WallArgs& W, cudaStream_t s);
cudaError_t launch_dt(const DtArgs& D, cudaStream_t s);
cudaError_t launch_sponge_mean(const SpongeArgs& S, int max_rows, cudaStream_t s);
cudaError_t launch_inflow(const InflowArgs& I, int Nj, int Nk, int ng, cudaStream_t s);

}  // namespace wm
