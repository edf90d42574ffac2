// Device-side descriptors shared by the kernels of libwmles_cuda.so.
//
// Every launch works on a *view*: a set of one or more independent cases whose blocks,
// per-case constants, wall faces and stage tiles are concatenated into device tables.
// Blocks carry a global index (into the view's block table) and their case's index.
#pragma once
#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/wmles_cuda.h"

namespace wm {

// runs `set` (a kernel attribute set-up, which holds for the current device only) once per
// device: `done` keeps one bit per device ordinal below 64 (others set it on every call); two
// threads racing on a device both set the same value
template <class F>
inline cudaError_t once_per_device(std::atomic<unsigned long long>& done, F set) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = dev >= 0 && dev < 64 ? 1ull << dev : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = set();
    if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

constexpr int MAX_CASES = WM_MAX_BLOCKS;   // a case has at least one block

// one structured block, resident in device memory
struct BlockDev {
    int n[3];          // interior cells
    int N[3];          // ghosted extents
    int ng;
    int case_id;       // index of the block's case in the view
    long long ncell;   // Ni*Nj*Nk
    long long plane;   // Nj*Nk
    const double* met;     // WM_NMET x ncell (float64)
    const float* met32;    // WM_NMET x ncell (float32 copy for the mixed form), may be null
    int wall[6];       // view wall index of face (axis*2 + side), -1 if not wall-modelled
};

// per-case physical constants, precomputed where the kernels only need a derived value
struct CaseDev {
    double gamma, Rg, Pr, Prt, mu_ref, T_ref, S_suth;
    double cp, gm1, inv_gm1, inv_Rg, inv_Tref, TrefS, inv_Pr, inv_Prt;
    double th0, inv_dth;   // Hybrid: s = clip((theta - th0) * inv_dth, 0, 1)
    double sgs_c;          // model coefficient
    double cfl, nu_fac;    // nu_fac = max(4/3, gamma/Pr)
    double Pr13, Pr3, kader_beta;   // Pr^(1/3), Pr^3, (3.85 Pr^(1/3) - 1.3)^2 + 2.12 ln Pr
    int cmf_dir;
    double cmf_target, cmf_volume;
    int sponge;
    double sp_xs, sp_inv_dx, sp_sigma0, sp_invL;   // sigma = sigma0 * ramp(eta)
    unsigned int* status;  // the case's status word (WM_ST_* bits, set with atomicOr)
};

struct WallDev {
    int block, axis, side, n_match;   // block: view block index
    int isothermal, n_iter;
    int nt1, nt2;              // tangential interior extents (axes in increasing order)
    double T_wall, kappa, B, ekb;
    const double* geom;        // 5 x nf
    double* F;                 // 5 x nf flux override (written by the wall kernel)
    double* tq;                // 2 x nf (tau_w, q_w)
};

// stage-kernel work item: one (j,k) tile of one block over planes [i0, i1)
struct Tile {
    int blk, j0, k0, i0, i1;   // blk: view block index
};

// one case's ghost-cell program inside a view-wide gather launch
struct GhostSeg {
    const int* dst;
    const int* src;
    const int* ops;
    const int* op_code;
    const double* op_nrm;
    const double* bc;          // the case's BC table (8 per BC)
    const double* inflow;      // 5 x inflow_n (or null)
    long long inflow_n;
    int start, count;          // entries [start, start + count) of the launch
    int block0;                // view index of the case's first block
    double gamma, gm1, Rg;
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
    const int* cta_first;         // CTA c runs tiles [cta_first[c], cta_first[c+1]); null: tile c
    int nctas;                    // grid size
    int stage;                    // 0: q_out = RHS; 1,2,3: SSP-RK3 stage
    int ncases;
    const int* case_slot_start;   // ncases + 1: partial-sum slots of case c are [start[c], start[c+1])
    double* cmf_part;             // stage 3 with constant mass flux: per (column, plane, warp) partials
    unsigned int* cmf_counter;    // last-CTA-done counter (the last CTA resets it)
    double* cmf_delta;            // per case: constant-mass-flux shift, written by the last CTA
    const double* dt[MAX_CASES];  // per case: device time step
    int cmf_slot_start[WM_MAX_BLOCKS];   // first partial-sum slot of each block
    StatePtrs p[WM_MAX_BLOCKS];
};

}  // namespace wm
