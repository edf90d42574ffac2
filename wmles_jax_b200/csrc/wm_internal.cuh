// Device-side descriptors shared by the kernels of libwmles_cuda.so.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/wmles_cuda.h"

namespace wm {

// one structured block of a case, resident in device memory
struct BlockDev {
    int n[3];          // interior cells
    int N[3];          // ghosted extents
    int ng;
    int case_id;       // index into the CaseDev table
    long long ncell;   // Ni*Nj*Nk
    long long plane;   // Nj*Nk
    const double* met;     // WM_NMET x ncell (float64)
    const float* met32;    // WM_NMET x ncell (float32 copy for the mixed form), may be null
    int wall[6];       // wall index of face (axis*2 + side), -1 if not wall-modelled
};

// per-case physical constants, precomputed where the kernels only need a derived value
struct CaseDev {
    double gamma, Rg, Pr, Prt, mu_ref, T_ref, S_suth;
    double cp, gm1, inv_gm1, inv_Rg, inv_Tref, TrefS, inv_Pr, inv_Prt;
    double th0, inv_dth;   // Hybrid: s = clip((theta - th0) * inv_dth, 0, 1)
    double sgs_c;          // model coefficient
    double cfl, nu_fac;    // nu_fac = max(4/3, gamma/Pr)
    int cmf_dir;
    double cmf_target, cmf_volume;
    int sponge;
    double sp_xs, sp_inv_dx, sp_sigma0, sp_invL;   // sigma = sigma0 * ramp(eta)
};

struct WallDev {
    int block, axis, side, n_match;
    int isothermal, n_iter;
    int nt1, nt2;              // tangential interior extents (axes in increasing order)
    double T_wall, kappa, B, ekb;
    const double* geom;        // 5 x nf
    double* F;                 // 5 x nf flux override (written by the wall kernel)
    double* tq;                // 2 x nf (tau_w, q_w)
};

// stage-kernel work item: one (j,k) tile of one block over planes [i0, i1)
struct Tile {
    int blk, j0, k0, i0, i1;
};

struct StatePtrs {
    const double* q_in;    // stage input (ghosts filled)
    const double* q0;      // Q at the start of the step (RK stages 2, 3)
    double* q_out;         // stage output (interior written)
    const double* spmean;  // sponge spanwise mean of q_in, 5 x Ni x Nj (or null)
};

// records the calling thread's error text (read by wm_last_error) and returns `code`
int set_error(int code, const char* msg);

struct StageArgs {
    const BlockDev* blocks;
    const CaseDev* cases;
    const WallDev* walls;
    const Tile* tiles;
    int ntiles;
    int stage;              // 0: q_out = RHS; 1,2,3: SSP-RK3 stage
    const double* dt;       // device time step (per case: dt[case_id])
    double* cmf_part;       // stage 3 with constant mass flux: per-tile partial sums
    unsigned int* cmf_counter;  // last-CTA-done counter (the last CTA resets it)
    double* cmf_delta;      // constant-mass-flux shift, written by the last CTA
    StatePtrs p[WM_MAX_BLOCKS];
};

}  // namespace wm
