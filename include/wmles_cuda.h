/*
 * wmles_cuda.h - C ABI of libwmles_cuda.so, the B200 (sm_100a) implementation of the
 * wmles explicit RHS + SSP-RK3 step.
 *
 * Plain C: raw pointers and sizes, no torch or CUDA types in the signatures (a stream is
 * passed as `void*` holding a cudaStream_t; NULL = legacy default stream).  Every entry
 * point returns 0 on success or a negative WM_E* status; wm_last_error() gives the text
 * of the calling thread's last error.  No C++ exception crosses this boundary.
 *
 * Ownership: a wm_case owns its device copies of the metrics, ghost programs, wall
 * geometry, work buffers (two RK stage states) and reduction scratch; it is created once
 * per Solver and freed by wm_case_destroy.  State arrays passed to the entry points are
 * borrowed device pointers (one per block, float64, layout (5, Ni, Nj, Nk) C-order with
 * Ni = ni + 2 ng ...), used only during the call on the given stream and never freed.
 *
 * Reference interfaces replaced (EduardoMolina/wmles_jax):
 *   wm_case_create   Solver.__init__            wmles/solver.py:40-51 (+ Mesh.finalize output)
 *   wm_apply_bcs     Solver.apply_bcs           wmles/solver.py:59-73
 *   wm_rhs           Solver.rhs / _rhs           wmles/solver.py:97-106,159-160
 *   wm_max_dt        Solver.max_dt / _dt         wmles/solver.py:135-154
 *   wm_advance       Solver.advance             wmles/solver.py:110-133,156-157
 *   wm_step          max_dt + advance, as the drivers call them (examples/channel_wmles.py:124-125)
 *   wm_wall_stats    Solver.wall_stats          wmles/solver.py:163-179
 *   wm_plane_stats   PlaneStats.accumulate      wmles/channel5200.py:121-152
 *   wm_derived_fields derived_fields            wmles/io_vtk.py:269-293
 *   wm_block_geometry Mesh.finalize metrics     wmles/mesh.py:53-73,213-242 (one block)
 */
#ifndef WMLES_CUDA_H
#define WMLES_CUDA_H

#ifdef __cplusplus
extern "C" {
#endif

#define WM_ABI_VERSION 1
#define WM_MAX_BLOCKS 96      /* blocks per case (all cases of one batched launch) */
#define WM_NMET 27            /* metric components per cell, see WM_MET_* */
#define WM_NDERIVED 11        /* derived output fields per cell, see wm_derived_fields */

/* status codes */
#define WM_OK 0
#define WM_E_INVALID (-1)     /* malformed descriptor or argument */
#define WM_E_CUDA (-2)        /* a CUDA runtime call failed */
#define WM_E_NONFINITE (-3)   /* non-finite or non-positive dt / state detected */
#define WM_E_UNSUPPORTED (-4) /* option not built into this library */

/* metric component order (per cell, float64): face area vector of the cell's LOWER face
 * in each direction (the reference's S[d][:, c] for face index c), volume, centre, the SGS
 * filter width V^(1/3), 1/V, and for the lower face in each direction the unit vector
 * e = (xc[c] - xc[c-1]) / |.| between the two cell centres and 1/|xc[c] - xc[c-1]| (the
 * geometry of the viscous face-gradient correction; zero on the first layer) */
enum { WM_MET_SIX = 0, WM_MET_SIY, WM_MET_SIZ, WM_MET_SJX, WM_MET_SJY, WM_MET_SJZ,
       WM_MET_SKX, WM_MET_SKY, WM_MET_SKZ, WM_MET_VOL, WM_MET_XCX, WM_MET_XCY, WM_MET_XCZ,
       WM_MET_DELTA, WM_MET_IVOL,
       WM_MET_EIX, WM_MET_EIY, WM_MET_EIZ, WM_MET_IDI,
       WM_MET_EJX, WM_MET_EJY, WM_MET_EJZ, WM_MET_IDJ,
       WM_MET_EKX, WM_MET_EKY, WM_MET_EKZ, WM_MET_IDK };

enum { WM_SCHEME_KEP = 0, WM_SCHEME_MUSCL = 1, WM_SCHEME_HYBRID = 2 };
enum { WM_LIMITER_ALBADA = 0, WM_LIMITER_MINMOD = 1 };
enum { WM_SGS_NONE = 0, WM_SGS_SMAGORINSKY = 1, WM_SGS_WALE = 2, WM_SGS_VREMAN = 3 };
enum { WM_PREC_FP64 = 0, WM_PREC_MIXED = 1 };

/* ghost-cell program: every listed ghost cell is a chain of per-cell maps applied to
 * one source value (an interior cell, an inflow value or a constant) */
enum { WM_SRC_CELL = 0, WM_SRC_INFLOW = 1, WM_SRC_CONST = 2 };
enum { WM_OP_SLIP = 1, WM_OP_NOSLIP = 2, WM_OP_FARFIELD = 3 };

typedef struct {
    double gamma, R, Pr, Pr_t, mu_ref, T_ref, S_suth;
} wm_gas;

typedef struct {
    int n[3];                 /* interior cells per direction */
    int ng;                   /* ghost layers (the reference's ng = 3) */
    const double* metrics;    /* WM_NMET x Ni x Nj x Nk, host or device memory (a device
                                 table, e.g. from wm_block_geometry, is copied on the device) */
} wm_block;

typedef struct {
    int block, axis, side;    /* the wall-modelled face */
    int n_match;              /* sample cell counted from the wall (1 = first cell) */
    int isothermal;           /* 0: adiabatic (recovery temperature, q_w = 0) */
    double T_wall;
    double kappa, B;
    int n_iter;               /* Newton iterations on Spalding's law */
    const double* geom;       /* host, 5 x nt1 x nt2: |S|, n_out (3), h; tangential axes
                                 in increasing order, interior extent */
} wm_wall;

typedef struct {
    int count;                /* ghost cells to write */
    const int* dst;           /* 2*count: block, flat cell index */
    const int* src;           /* 2*count: (kind << 24) | block (or BC id for CONST), flat index */
    const int* ops;           /* 2*count: first op, number of ops (applied in order) */
    int nops;
    const int* op_code;       /* nops: code | (bc id << 8) | (side << 16) */
    const double* op_nrm;     /* 3*nops: unit normal of the boundary face */
} wm_ghost_program;

typedef struct {
    int block;                /* i-min face of this block; at most 2048 cells along k with
                                 ghosts (wider: WM_E_UNSUPPORTED at creation) */
    int n_modes, n_tab;
    const double* modes;      /* host, 3 x 4 x n_modes: kx, ky, kz, phase per component */
    const double* table;      /* host, n_tab x 7: y/L, U, V, uu, vv, ww, uv (by U_inf) */
    double U_inf, L, rho_inf, p_inf;
} wm_inflow;

typedef struct {
    int enabled;
    double x_start_l, x_end_l, strength, U_inf, L;
} wm_sponge;

typedef struct {
    wm_gas gas;
    int scheme;               /* WM_SCHEME_* */
    int kep_order;            /* 2 or 4 (central flux of KEP and of Hybrid) */
    int limiter;              /* WM_LIMITER_* (MUSCL and Hybrid) */
    double th0, th1;          /* Hybrid switch thresholds */
    int sgs;                  /* WM_SGS_* */
    double sgs_coeff;         /* Cs, Cw or Cs (Vreman) */
    double cfl;
    int precision;            /* WM_PREC_* */
    int cmf_dir;              /* ConstantMassFlux direction, -1 = none */
    double cmf_target;
    double cmf_volume;        /* sum of interior volumes, as the reference sums them */
    int nblocks;
    const wm_block* blocks;
    int nwalls;
    const wm_wall* walls;
    int nbc;
    const double* bc_table;   /* 8 per BC: const state / prim_inf (5), T_wall, isothermal, 0 */
    wm_ghost_program ghost_rhs;   /* ghost cells read by the RHS */
    wm_ghost_program ghost_all;   /* every ghost cell (apply_bcs) */
    const wm_inflow* inflow;      /* NULL if no synthetic-turbulence inflow */
    wm_sponge sponge;
    int tile;                 /* stage-kernel tile shape id (0 = 8x32, 1 = 16x16, 2 = 4x32,
                                 3 = 16x32, mixed form only); -1 = automatic: 0 for FP64,
                                 3 for the mixed form */
    int chunk;                /* planes per CTA along i, 0 = automatic */
} wm_case_desc;

typedef struct wm_case wm_case;

int wm_version(void);
const char* wm_last_error(void);

int wm_case_create(const wm_case_desc* desc, wm_case** out);
void wm_case_destroy(wm_case* c);

/* Fill every ghost cell of q (in place) at `time`. */
int wm_apply_bcs(wm_case* c, double* const* q, double time, void* stream);

/* r = RHS(q) on the interior (ghost cells of r are left untouched); fills the ghost
 * cells of q it reads, in place. */
int wm_rhs(wm_case* c, double* const* q, double* const* r, double time, void* stream);

/* CFL time step of q, written to dt_dev (device double).  Interior only; q is not
 * modified. */
int wm_max_dt(wm_case* c, const double* const* q, double* dt_dev, void* stream);

/* One SSP-RK3 step (plus the case's constraint) of q_in with the device time step
 * *dt_dev, written to q_out (interior).  Ghost cells of q_in are refreshed in place. */
int wm_advance(wm_case* c, double* const* q_in, double* const* q_out, const double* dt_dev,
               double time, void* stream);

/* dt = max_dt(q_in) written to dt_dev, then advance(q_in -> q_out, dt). */
int wm_step(wm_case* c, double* const* q_in, double* const* q_out, double* dt_dev,
            double time, void* stream);

/* One step with a given time step *dt_in (= wm_max_dt(q_in)), fused with the next step's
 * CFL reduction: after the constraint pass *dt_next = max_dt(q_out).  A driver loop calls
 * wm_max_dt once, then feeds each call's dt_next to the next call (the reference's loop
 * examples/channel_wmles.py:124-125 with one reduction pass per step instead of two). */
int wm_step_fused(wm_case* c, double* const* q_in, double* const* q_out, const double* dt_in,
                  double* dt_next, double time, void* stream);

/* CFL time step of a multiblock state with no device allocation (no counterpart in the
 * reference: it exists for callers that cannot allocate device memory, e.g. code running
 * inside another framework's memory pool or a fixed device-memory budget, and it needs no
 * wm_case).  dims: 4 ints per block (ni, nj, nk, ng); q[b], metrics[b]: device arrays of
 * block b ((5, Ni, Nj, Nk) state, (WM_NMET, Ni, Nj, Nk) metrics, see WM_MET_*); dt_dev:
 * device double.  Its reduction scratch is a file-scope static device array of
 * WM_NOALLOC_MAX_PARTIALS slots (one per 256 interior cells, so at most
 * WM_NOALLOC_MAX_PARTIALS * 256 interior cells in total; larger inputs are rejected with
 * WM_E_INVALID).  The first call on a device looks the array up (cudaGetSymbolAddress), so
 * make it before any stream capture; the lookup is repeated only if the device's context
 * has been replaced since (cudaDeviceReset), and a first call after that replacement must
 * also come before any capture.  All calls share the array: calls that overlap on the GPU
 * race and must be serialised by the caller. */
#define WM_NOALLOC_MAX_PARTIALS 32768
int wm_max_dt_noalloc(int nblocks, const int* dims, const double* const* q, const double* const* metrics,
                      const wm_gas* gas, double cfl, double* dt_dev, void* stream);

/* Per-case status word (no reference counterpart: the reference only prints rho_min,
 * examples/channel_wmles.py:141).  The kernels OR these bits into the case's word as they
 * see the condition; the word keeps them until it is cleared:
 *   WM_ST_NONFINITE   a NaN or infinite conservative value in a state the CFL / constraint
 *                     pass reads (a step's output, or the input of wm_max_dt)
 *   WM_ST_RHO         density <= 0 there
 *   WM_ST_PRESSURE    pressure <= 0 there
 *   WM_ST_DT          a CFL time step that is not finite and positive
 *   WM_ST_WALL        a wall-model Newton solve still moving (relative update > 1e-8) after
 *                     its n_iter iterations (informational: the reference stops there too)
 * WM_ST_FATAL = the first four: the state is no longer a flow state. */
#define WM_ST_NONFINITE 1u
#define WM_ST_RHO 2u
#define WM_ST_PRESSURE 4u
#define WM_ST_DT 8u
#define WM_ST_WALL 16u
#define WM_ST_FATAL (WM_ST_NONFINITE | WM_ST_RHO | WM_ST_PRESSURE | WM_ST_DT)

/* Read the case's status word into *status (synchronises `stream`); clear != 0 resets it. */
int wm_case_status(wm_case* c, unsigned* status, int clear, void* stream);

/* WM_E_NONFINITE (with the bits named in wm_last_error) if the case's status word holds a
 * WM_ST_FATAL bit, else WM_OK; synchronises `stream` and clears the word. */
int wm_check(wm_case* c, void* stream);

/* (tau_w, q_w) of every wall-modelled face: out[w] is a device buffer of 2 x nt1 x nt2. */
int wm_wall_stats(wm_case* c, const double* const* q, double* const* out, void* stream);

/* Plane statistics of block `block` (PlaneStats.accumulate, wmles/channel5200.py:121-152):
 * for every interior j-plane, the means over interior (i, k) of rho, u, v, w, uu, vv, ww, uv,
 * uw, vw, T and p are ADDED to sum (device, 12 x nj doubles, quantity-major), so a driver
 * samples the flow on the device; q is the block's state (ghost cells are not read).  The
 * block must have the same y on every (i, k) of a plane (an unskewed channel block), as in
 * the reference. */
int wm_plane_stats(wm_case* c, int block, const double* q, double* sum, void* stream);

/* Derived output fields of every block (derived_fields, wmles/io_vtk.py:269-293): out[b] is
 * a device array of WM_NDERIVED x ni x nj x nk doubles (interior only) receiving rho, u, v,
 * w, p, T, Mach number, SGS viscosity mu_t, molecular viscosity mu, vorticity magnitude and
 * Q-criterion.  q must have its first ghost layer filled (call wm_apply_bcs first, as the
 * reference does); it is not modified. */
int wm_derived_fields(wm_case* c, const double* const* q, double* const* out, void* stream);

/* Geometry of one block on the device (the metrics of Mesh.finalize, wmles/mesh.py:53-73,
 * for one block whose ghost nodes are filled, wmles/mesh.py:213-242), with the host path's
 * arithmetic: every output bit-identical to it except the filter width V^(1/3) of the
 * packed table (device pow; within a few ulp).  N: cells per direction including ghosts
 * (n + 2 ng).  Device float64 arrays, C order: X 3 x (N0+1) x (N1+1) x (N2+1) nodes;
 * vol N0 x N1 x N2; xc 3 x N0 x N1 x N2; S[d], xf[d] 3 x (N0 + (d==0)) x (N1 + (d==1)) x
 * (N2 + (d==2)) face area vectors and face centres along +d; met (NULL: not written)
 * WM_NMET x N0 x N1 x N2, the packed table wm_block.metrics takes.  Asynchronous on the
 * stream; allocates nothing. */
int wm_block_geometry(const double* X, const int* N, double* vol, double* xc, double* const* S,
                      double* const* xf, double* met, void* stream);

/* Batched stepping of several resident cases (no reference counterpart: the reference
 * advances one case per Solver).  A wm_batch is a fixed set of cases that share the
 * precision, scheme, SGS model and tile shape; wm_batch_step advances all of them by one
 * fused step (as wm_step_fused) with ONE launch per kernel per RK stage, so its launch count
 * does not grow with the number of cases.  Every per-case reduction (CFL minimum, constant
 * mass flux) runs over that case's own cells in a fixed order, so a case's result is
 * bit-identical whether it is stepped alone (wm_step_fused) or in any batch.
 *   q_in, q_out: per block of the batch, the member cases' blocks in member order;
 *   dt_in, dt_next: per case, device doubles; times: per case, host doubles.
 * The batch holds pointers to its members: destroy it before any of them.  A case's own
 * entries and every batch holding it use the case's work states, so calls that touch one
 * case must be ordered (one stream, or events).  With no member carrying a synthetic
 * inflow the launches depend only on the pointers, so a step can be captured in a CUDA
 * graph and replayed while the same buffers alternate. */
typedef struct wm_batch wm_batch;
int wm_batch_create(int ncases, wm_case* const* cases, wm_batch** out);
void wm_batch_destroy(wm_batch* b);
int wm_batch_step(wm_batch* b, double* const* q_in, double* const* q_out, const double* const* dt_in,
                  double* const* dt_next, const double* times, void* stream);
/* Status words of the batch's member cases, in member order, copied to status (ncases
 * unsigned, host memory; page-locked memory keeps the copy asynchronous) on `stream`
 * without waiting: read them after an event recorded behind this call.  The words are not
 * cleared (their bits only accumulate), so a later read never loses a fault. */
int wm_batch_status(wm_batch* b, unsigned* status, void* stream);
/* blocks and stage tiles of the batch, and the number of kernel launches of one step */
int wm_batch_info(wm_batch* b, int* nblocks, int* ntiles, long long* launches_per_step);

/* Launch accounting and device timing of this library's kernels.  kind: WM_KIND_*.
 * wm_profile_enable(c, 1) resets the counters and starts recording a CUDA event pair around
 * every launch on the launching stream; wm_profile_read waits for the recorded events and
 * returns the summed device time (ms) and the launch count of one kind (-1 = all kinds;
 * launch counts are kept even with timing disabled).  No reference counterpart: this is the
 * measurement hook of the benchmark.  Kinds: STAGE the fused RHS + RK stage kernel; GHOST
 * the surface launch before each stage (ghost cells, wall-model flux overrides, sponge
 * means) and the ghost fill of wm_apply_bcs; WALL the wall model of wm_wall_stats; DT the
 * CFL / constraint pass; SOURCE the synthetic-inflow fill. */
enum { WM_KIND_STAGE = 0, WM_KIND_GHOST = 1, WM_KIND_WALL = 2, WM_KIND_DT = 3, WM_KIND_SOURCE = 4,
       WM_NKINDS = 5 };
int wm_profile_enable(wm_case* c, int enable);
int wm_profile_read(wm_case* c, int kind, double* ms_total, long long* launches);

#ifdef __cplusplus
}
#endif
#endif /* WMLES_CUDA_H */
