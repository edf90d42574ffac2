// Argument blocks and launchers of the surface and reduction kernels.
#pragma once
#include "wm_internal.cuh"

namespace wm {

struct GhostArgs {
    int count;
    const int* dst;
    const int* src;
    const int* ops;
    const int* op_code;
    const double* op_nrm;
    const double* bc;         // 8 per BC
    const double* inflow;     // 5 x inflow_n (or null)
    long long inflow_n;
    double* stash;            // non-null: two-phase gather/scatter (5 x count)
    double gamma, gm1, Rg;
    double* q[WM_MAX_BLOCKS];
    long long ncell[WM_MAX_BLOCKS];
};

struct WallArgs {
    const BlockDev* blocks;
    const CaseDev* cases;
    WallDev* walls;
    int nwalls;
    int max_faces;
    double Pr13;          // Pr^(1/3)
    double Pr3;           // Pr^3
    double kader_beta;    // (3.85 Pr^(1/3) - 1.3)^2 + 2.12 ln Pr
    const double* q[WM_MAX_BLOCKS];
};

struct DtArgs {
    const BlockDev* blocks;
    const CaseDev* cases;
    int nblocks;
    int ctas_per_block;
    double* q[WM_MAX_BLOCKS];      // state (modified in place when cmf is applied)
    const double* cmf_delta;       // constant-mass-flux shift from stage 3 (null: none)
    int want_dt;                   // 0: constraint only
    double* dt_part;               // per-CTA minima
    unsigned int* counter;         // last-CTA-done counter (reset by the last CTA)
    double* dt_out;                // dt of the case
};

struct SpongeArgs {
    const BlockDev* blocks;
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
    double* out;             // 5 x (ng * Nj * Nk)
};

cudaError_t launch_ghost(const GhostArgs& G, cudaStream_t s);
cudaError_t launch_wall(const WallArgs& W, cudaStream_t s);
cudaError_t launch_dt(const DtArgs& D, cudaStream_t s);
cudaError_t launch_sponge_mean(const SpongeArgs& S, int max_rows, cudaStream_t s);
cudaError_t launch_inflow(const InflowArgs& I, int Nj, int Nk, int ng, cudaStream_t s);

}  // namespace wm
