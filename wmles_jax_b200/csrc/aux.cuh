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
    // ghost cells of q (a step's output): set to those of q_src (the step's input, as its
    // boundary fill left them) plus the constraint's shift, the reference's RK combination
    // of ghost values the RHS leaves at zero; ngcta = 0: ghost cells untouched
    const double* q_src[WM_MAX_BLOCKS];
    int ngcta;
    int gcta_start[WM_MAX_BLOCKS + 1];     // ghost-cell chunks of block b
    const double* cmf_delta;       // per case: constant-mass-flux shift from stage 3 (null: none)
    int want_dt;                   // 0: constraint only
    int met32;                     // read the float metric copy (mixed form)
    unsigned long long* dt_key;    // per case: running minimum as an order-preserving key
                                   // (DT_KEY_EMPTY between calls: reset by the last CTA)
    unsigned int* counter;         // last-CTA-done counter (reset by the last CTA)
    double* dt_out[MAX_CASES];     // per case: time step
};

// ghost cells of a block: every cell with an index outside the interior in some direction
__host__ __device__ inline long long ghost_cells(const BlockDev& B) {
    return B.ncell - (long long)B.n[0] * B.n[1] * B.n[2];
}

// flat index of ghost cell g (0 <= g < ghost_cells(B)), enumerated as the ghost planes
// i < ng, i >= ng + ni (all j, k), then for interior i the ghost rows in j (all k), then for
// interior (i, j) the ghost cells in k
__device__ __forceinline__ long long ghost_cell_index(const BlockDev& B, long long g) {
    const int ng = B.ng, ni = B.n[0], nj = B.n[1], nk = B.n[2], Nj = B.N[1], Nk = B.N[2];
    const long long a = 2LL * ng * Nj * Nk;
    if (g < a) {
        const int p = int(g / ((long long)Nj * Nk));
        const long long r = g - (long long)p * Nj * Nk;
        const int i = p < ng ? p : ni + p;
        return (long long)i * Nj * Nk + r;
    }
    g -= a;
    const long long b = (long long)ni * 2 * ng * Nk;
    if (g < b) {
        const int ii = int(g / (2LL * ng * Nk));
        const int r = int(g - (long long)ii * 2 * ng * Nk);
        const int p = r / Nk, k = r - p * Nk;
        const int j = p < ng ? p : nj + p;
        return ((long long)(ng + ii) * Nj + j) * Nk + k;
    }
    g -= b;
    const long long t = g / (2 * ng);
    const int p = int(g - t * 2 * ng);
    const int ii = int(t / nj), jj = int(t - (long long)ii * nj);
    const int k = p < ng ? p : nk + p;
    return ((long long)(ng + ii) * Nj + (ng + jj)) * Nk + k;
}

// key of DBL_MAX, the value of an empty minimum (the reset value of DtArgs::dt_key)
constexpr unsigned long long DT_KEY_EMPTY = 0xFFEFFFFFFFFFFFFFull;

struct SpongeArgs {
    const BlockDev* blocks;
    const CaseDev* cases;
    int nblocks;
    int nrows;                     // rows that reach into a sponge, over the view's blocks
    const int* rows;               // nrows x (view block, interior row (i - ng) * nj + (j - ng))
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
    const double* prof;      // 6 x (ng * Nj * Nk): the time-independent profile factors per ghost cell
    const double* cz;        // extruded plane: cos(kz z), then sin(kz z), each 3 x n_modes x Nk;
                             // null: general plane (direct cosines)
};

// partial mode sums per (component, cell) of the synthetic inflow (contiguous mode ranges)
constexpr int IN_PARTS = 4;
// kernel launches of one inflow fill (mode sums, then the rows)
constexpr int IN_LAUNCHES = 2;
// the rows' launch: one warp per velocity component of a ghost row; the row's three noise
// fields sit in the launch's default shared memory (48 KB), which bounds the ghosted span
constexpr int IN_ROW_NT = 96;
constexpr int IN_ROW_MAX_NK = 48 * 1024 / (3 * 8);
// extruded plane: ghost rows per CTA of the mode sums, threads per CTA, and the largest
// dynamic shared memory of that launch (one component's cos / sin (kz z) table and the rows'
// sincos of alpha)
constexpr int IN_EXT_ROWS = 4, IN_EXT_NT = 256;
constexpr size_t inflow_ext_smem_max() { return 200 * 1024; }
size_t inflow_ext_smem(int n_modes, int Nk);

// before each stage kernel: ghost gather (single phase), wall model and sponge means in one
// launch; the CTA counts are filled in by the launcher (an empty part has none)
struct SurfaceArgs {
    GhostArgs G;
    WallArgs W;
    SpongeArgs S;          // nblocks = 0: no sponge
    int g_ctas, w_per, w_ctas, s_ctas;
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
cudaError_t launch_surface(SurfaceArgs& A, cudaStream_t s);
cudaError_t launch_wall(const WallArgs& W, cudaStream_t s);
cudaError_t launch_dt(const DtArgs& D, cudaStream_t s);
cudaError_t launch_status_gather(const CaseDev* cases, int ncases, unsigned* out, cudaStream_t s);
// set-up: flags[row] = 1 for the interior (i, j) rows of a block with a cell inside the
// sponge (xcx: the block's cell-centre x metric; invL, xs, inv_dx: the case's sponge constants)
cudaError_t launch_sponge_flags(const double* xcx, long long plane, int Nk, int ng, int ni, int nj, int nk,
                                double invL, double xs, double inv_dx, unsigned char* flags, cudaStream_t s);
cudaError_t launch_inflow(const InflowArgs& I, int Nj, int Nk, int ng, cudaStream_t s);
// set-up of a case's inflow: prof (always) and, for an extruded plane, cz (I.prof, I.cz are
// the destinations here)
cudaError_t launch_inflow_setup(const InflowArgs& I, int Nj, int Nk, int ng, double* prof, double* cz, cudaStream_t s);

}  // namespace wm
