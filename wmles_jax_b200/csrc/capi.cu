// C ABI of libwmles_cuda.so (include/wmles_cuda.h): case set-up and step orchestration.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "wm_internal.cuh"
#include "stage.cuh"
#include "aux.cuh"

using namespace wm;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                             \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(WM_E_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),   \
                        __FILE__, __LINE__);                                                 \
    } while (0)

struct GhostProg {
    int count = 0;
    int *dst = nullptr, *src = nullptr, *ops = nullptr, *op_code = nullptr;
    double* op_nrm = nullptr;
};

}  // namespace

namespace wm {
int set_error(int code, const char* msg) {
    g_err = msg;
    return code;
}
}  // namespace wm

struct wm_case {
    int device = 0;
    int nblocks = 0;
    std::vector<BlockDev> hb;           // host copies of the block descriptors
    std::vector<void*> allocs;
    BlockDev* d_blocks = nullptr;
    CaseDev hc{};
    CaseDev* d_case = nullptr;
    std::vector<WallDev> hw;
    WallDev* d_walls = nullptr;
    int max_wall_faces = 0;
    std::vector<Tile> tiles;
    Tile* d_tiles = nullptr;
    StageOpts opts{};
    std::vector<double*> work[2];
    GhostProg prog_rhs, prog_all;
    double* stash = nullptr;
    double* d_bc = nullptr;
    bool has_inflow = false;
    int inflow_block = -1;
    double *d_modes = nullptr, *d_table = nullptr, *inflow_buf = nullptr;
    wm_inflow inflow{};
    long long inflow_n = 0;
    bool sponge = false;
    std::vector<double*> spmean;
    int sponge_rows = 0;
    double *d_cmf_part = nullptr, *d_dt_part = nullptr, *d_dt_tmp = nullptr, *d_cmf_delta = nullptr;
    unsigned* d_counter = nullptr;       // [0]: CFL reduction, [1]: constant-mass-flux reduction
    int dt_ctas = 0;
    double Pr13 = 0, Pr3 = 0, kader_beta = 0;
    // launch accounting / event timing (wm_profile_*)
    long long nlaunch[WM_NKINDS] = {0, 0, 0, 0, 0};
    bool prof = false;
    struct Rec { int kind; cudaEvent_t a, b; };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
};

namespace {

template <typename T>
int dev_alloc(wm_case* c, T** p, size_t count) {
    void* v = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(&v, sizeof(T) * count);
    if (e != cudaSuccess) return fail(WM_E_CUDA, "cudaMalloc(%zu bytes): %s", sizeof(T) * count, cudaGetErrorString(e));
    c->allocs.push_back(v);
    *p = static_cast<T*>(v);
    return WM_OK;
}

template <typename T>
int dev_upload(wm_case* c, T** p, const T* host, size_t count) {
    int r = dev_alloc(c, p, count);
    if (r) return r;
    if (count && host) CK(cudaMemcpy(*p, host, sizeof(T) * count, cudaMemcpyHostToDevice));
    return WM_OK;
}

cudaEvent_t pool_event(wm_case* c) {
    if (!c->pool.empty()) {
        cudaEvent_t e = c->pool.back();
        c->pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// brackets one launch of `kind`: counts it and, when profiling, records an event pair
struct LaunchScope {
    wm_case* c;
    int kind, slot = -1;
    cudaStream_t s;
    LaunchScope(wm_case* c_, int kind_, cudaStream_t s_, int n = 1) : c(c_), kind(kind_), s(s_) {
        c->nlaunch[kind] += n;
        if (c->prof) {
            wm_case::Rec r{kind, pool_event(c), pool_event(c)};
            cudaEventRecord(r.a, s);
            c->recs.push_back(r);
            slot = (int)c->recs.size() - 1;
        }
    }
    ~LaunchScope() {
        if (slot >= 0) cudaEventRecord(c->recs[slot].b, s);
    }
};

int upload_prog(wm_case* c, GhostProg* g, const wm_ghost_program& p) {
    g->count = p.count;
    int r;
    if ((r = dev_upload(c, &g->dst, p.dst, 2 * (size_t)p.count))) return r;
    if ((r = dev_upload(c, &g->src, p.src, 2 * (size_t)p.count))) return r;
    if ((r = dev_upload(c, &g->ops, p.ops, 2 * (size_t)p.count))) return r;
    if ((r = dev_upload(c, &g->op_code, p.op_code, (size_t)p.nops))) return r;
    if ((r = dev_upload(c, &g->op_nrm, p.op_nrm, 3 * (size_t)p.nops))) return r;
    return WM_OK;
}

int validate(const wm_case_desc* d) {
    if (!d) return fail(WM_E_INVALID, "null descriptor");
    if (d->nblocks < 1 || d->nblocks > WM_MAX_BLOCKS)
        return fail(WM_E_INVALID, "nblocks=%d outside [1, %d]", d->nblocks, WM_MAX_BLOCKS);
    if (d->scheme < 0 || d->scheme > WM_SCHEME_HYBRID) return fail(WM_E_INVALID, "unknown scheme %d", d->scheme);
    if (d->kep_order != 2 && d->kep_order != 4) return fail(WM_E_INVALID, "kep_order must be 2 or 4");
    if (d->sgs < 0 || d->sgs > WM_SGS_VREMAN) return fail(WM_E_INVALID, "unknown sgs %d", d->sgs);
    if (d->precision != WM_PREC_FP64 && d->precision != WM_PREC_MIXED)
        return fail(WM_E_INVALID, "unknown precision %d", d->precision);
    if (d->tile < -1 || d->tile > 3) return fail(WM_E_INVALID, "unknown tile shape %d", d->tile);
    if (d->tile == 3 && d->precision == WM_PREC_FP64)
        return fail(WM_E_UNSUPPORTED, "tile 3 (16x32) is built for the mixed form only");
    for (int b = 0; b < d->nblocks; ++b) {
        const wm_block& B = d->blocks[b];
        if (B.ng != 3) return fail(WM_E_UNSUPPORTED, "block %d: ng=%d (this build supports ng=3)", b, B.ng);
        for (int a = 0; a < 3; ++a)
            if (B.n[a] < B.ng) return fail(WM_E_INVALID, "block %d: n[%d]=%d < ng", b, a, B.n[a]);
        if (!B.metrics) return fail(WM_E_INVALID, "block %d: null metrics", b);
    }
    for (int w = 0; w < d->nwalls; ++w) {
        const wm_wall& W = d->walls[w];
        if (W.block < 0 || W.block >= d->nblocks || W.axis < 0 || W.axis > 2 || W.side < 0 || W.side > 1)
            return fail(WM_E_INVALID, "wall %d: bad block/axis/side", w);
        const int n = d->blocks[W.block].n[W.axis];
        if (W.n_match < 1 || W.n_match > n) return fail(WM_E_INVALID, "wall %d: n_match=%d", w, W.n_match);
    }
    if (d->cmf_dir >= 0 && !(d->cmf_volume > 0)) return fail(WM_E_INVALID, "cmf_volume must be positive");
    return WM_OK;
}

int choose_chunk(wm_case* c, int tj, int tk, int requested) {
    if (requested > 0) return requested;
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int occ = stage_ctas_per_sm(c->opts);
    if (occ < 1) occ = 1;
    const long long slots = (long long)sms * occ;
    int nimax = 0;
    long long jk = 0;
    for (const BlockDev& B : c->hb) {
        nimax = std::max(nimax, B.n[0]);
    }
    double best = 1e300;
    int best_ic = nimax;
    for (int ic = 4; ic <= std::max(4, nimax); ++ic) {
        long long ctas = 0;
        for (const BlockDev& B : c->hb) {
            jk = (long long)((B.n[1] + tj - 1) / tj) * ((B.n[2] + tk - 1) / tk);
            ctas += jk * ((B.n[0] + ic - 1) / ic);
        }
        const long long waves = (ctas + slots - 1) / slots;
        const double cost = double(waves) * (std::min(ic, nimax) + 3);
        if (cost < best - 1e-9) { best = cost; best_ic = ic; }
    }
    return best_ic;
}

void build_tiles(wm_case* c, int tj, int tk, int ic) {
    c->tiles.clear();
    for (int b = 0; b < c->nblocks; ++b) {
        const BlockDev& B = c->hb[b];
        const int ng = B.ng;
        for (int i0 = ng; i0 < ng + B.n[0]; i0 += ic)
            for (int j0 = ng; j0 < ng + B.n[1]; j0 += tj)
                for (int k0 = ng; k0 < ng + B.n[2]; k0 += tk)
                    c->tiles.push_back(Tile{b, j0, k0, i0, std::min(i0 + ic, ng + B.n[0])});
    }
}

GhostArgs ghost_args(wm_case* c, const GhostProg& g, double* const* q, bool two_phase) {
    GhostArgs G{};
    G.count = g.count;
    G.dst = g.dst; G.src = g.src; G.ops = g.ops; G.op_code = g.op_code; G.op_nrm = g.op_nrm;
    G.bc = c->d_bc;
    G.inflow = c->inflow_buf;
    G.inflow_n = c->inflow_n;
    G.stash = two_phase ? c->stash : nullptr;
    G.gamma = c->hc.gamma; G.gm1 = c->hc.gm1; G.Rg = c->hc.Rg;
    for (int b = 0; b < c->nblocks; ++b) { G.q[b] = q[b]; G.ncell[b] = c->hb[b].ncell; }
    return G;
}

int fill_inflow(wm_case* c, double time0, double time_dt, const double* dt, cudaStream_t s) {
    if (!c->has_inflow) return WM_OK;
    const BlockDev& B = c->hb[c->inflow_block];
    InflowArgs I{};
    I.block = c->d_blocks + c->inflow_block;
    I.modes = c->d_modes; I.table = c->d_table;
    I.n_modes = c->inflow.n_modes; I.n_tab = c->inflow.n_tab;
    I.U_inf = c->inflow.U_inf; I.L = c->inflow.L; I.rho_inf = c->inflow.rho_inf; I.p_inf = c->inflow.p_inf;
    I.gm1 = c->hc.gm1;
    I.time0 = time0; I.time_dt = time_dt; I.dt = dt;
    I.out = c->inflow_buf;
    LaunchScope ls(c, WM_KIND_SOURCE, s);
    CK(launch_inflow(I, B.N[1], B.N[2], B.ng, s));
    return WM_OK;
}

// one RHS evaluation fused with RK stage `stage` (0 = plain RHS)
int run_stage(wm_case* c, int stage, double* const* q_in, const double* const* q0, double* const* q_out,
              const double* dt, double time0, double time_dt, cudaStream_t s) {
    int r;
    if ((r = fill_inflow(c, time0, time_dt, dt, s))) return r;
    {
        LaunchScope ls(c, WM_KIND_GHOST, s, c->prog_rhs.count ? 1 : 0);
        CK(launch_ghost(ghost_args(c, c->prog_rhs, q_in, false), s));
    }
    if (!c->hw.empty()) {
        WallArgs W{};
        W.blocks = c->d_blocks; W.cases = c->d_case; W.walls = c->d_walls;
        W.nwalls = (int)c->hw.size(); W.max_faces = c->max_wall_faces;
        W.Pr13 = c->Pr13; W.Pr3 = c->Pr3; W.kader_beta = c->kader_beta;
        for (int b = 0; b < c->nblocks; ++b) W.q[b] = q_in[b];
        LaunchScope ls(c, WM_KIND_WALL, s);
        CK(launch_wall(W, s));
    }
    if (c->sponge) {
        SpongeArgs S{};
        S.blocks = c->d_blocks; S.nblocks = c->nblocks;
        for (int b = 0; b < c->nblocks; ++b) { S.q[b] = q_in[b]; S.mean[b] = c->spmean[b]; }
        LaunchScope ls(c, WM_KIND_SOURCE, s);
        CK(launch_sponge_mean(S, c->sponge_rows, s));
    }
    StageArgs A{};
    A.blocks = c->d_blocks; A.cases = c->d_case; A.walls = c->d_walls;
    A.tiles = c->d_tiles; A.ntiles = (int)c->tiles.size();
    A.stage = stage; A.dt = dt;
    A.cmf_part = (stage == 3 && c->hc.cmf_dir >= 0) ? c->d_cmf_part : nullptr;
    A.cmf_counter = c->d_counter + 1;
    A.cmf_delta = c->d_cmf_delta;
    for (int b = 0; b < c->nblocks; ++b) {
        A.p[b].q_in = q_in[b];
        A.p[b].q0 = q0 ? q0[b] : q_in[b];
        A.p[b].q_out = q_out[b];
        A.p[b].spmean = c->sponge ? c->spmean[b] : nullptr;
    }
    LaunchScope ls(c, WM_KIND_STAGE, s);
    CK(launch_stage(A, c->opts, s));
    return WM_OK;
}

int run_dt(wm_case* c, double* const* q, bool apply_cmf, bool want_dt, double* dt_out, cudaStream_t s) {
    DtArgs D{};
    D.blocks = c->d_blocks; D.cases = c->d_case; D.nblocks = c->nblocks;
    D.ctas_per_block = c->dt_ctas;
    for (int b = 0; b < c->nblocks; ++b) D.q[b] = q[b];
    D.cmf_delta = apply_cmf ? c->d_cmf_delta : nullptr;
    D.want_dt = want_dt ? 1 : 0;
    D.dt_part = c->d_dt_part; D.counter = c->d_counter;
    D.dt_out = dt_out ? dt_out : c->d_dt_tmp;
    LaunchScope ls(c, WM_KIND_DT, s);
    CK(launch_dt(D, s));
    return WM_OK;
}

}  // namespace

extern "C" {

int wm_version(void) { return WM_ABI_VERSION; }
const char* wm_last_error(void) { return g_err.c_str(); }

void wm_case_destroy(wm_case* c) {
    if (!c) return;
    for (auto& r : c->recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (cudaEvent_t e : c->pool) cudaEventDestroy(e);
    for (void* p : c->allocs) cudaFree(p);
    delete c;
}

int wm_case_create(const wm_case_desc* d, wm_case** out) {
    if (!out) return fail(WM_E_INVALID, "null output handle");
    *out = nullptr;
    int r = validate(d);
    if (r) return r;
    wm_case* c = new wm_case();
    auto bail = [&](int code) { wm_case_destroy(c); return code; };
    CK(cudaGetDevice(&c->device));
    c->nblocks = d->nblocks;

    // ---- physical constants
    const wm_gas& g = d->gas;
    CaseDev& C = c->hc;
    C.gamma = g.gamma; C.Rg = g.R; C.Pr = g.Pr; C.Prt = g.Pr_t; C.mu_ref = g.mu_ref; C.T_ref = g.T_ref;
    C.S_suth = g.S_suth;
    C.gm1 = g.gamma - 1.0;
    C.cp = g.gamma * g.R / C.gm1;
    C.inv_gm1 = 1.0 / C.gm1; C.inv_Rg = 1.0 / g.R; C.inv_Tref = 1.0 / g.T_ref;
    C.TrefS = g.T_ref + g.S_suth; C.inv_Pr = 1.0 / g.Pr; C.inv_Prt = 1.0 / g.Pr_t;
    C.th0 = d->th0; C.inv_dth = 1.0 / (d->th1 - d->th0);
    C.sgs_c = d->sgs_coeff;
    C.cfl = d->cfl;
    C.nu_fac = std::max(4.0 / 3.0, g.gamma / g.Pr);
    C.cmf_dir = d->cmf_dir; C.cmf_target = d->cmf_target; C.cmf_volume = d->cmf_volume;
    C.sponge = d->sponge.enabled;
    if (C.sponge) {
        C.sp_xs = d->sponge.x_start_l;
        C.sp_inv_dx = 1.0 / (d->sponge.x_end_l - d->sponge.x_start_l);
        C.sp_sigma0 = d->sponge.strength * d->sponge.U_inf / d->sponge.L;
        C.sp_invL = 1.0 / d->sponge.L;
    }
    c->Pr13 = std::pow(g.Pr, 1.0 / 3.0);
    c->Pr3 = std::pow(g.Pr, 3.0);
    c->kader_beta = std::pow(3.85 * std::pow(g.Pr, 1.0 / 3.0) - 1.3, 2.0) + 2.12 * std::log(g.Pr);
    c->opts = StageOpts{d->precision, d->scheme, d->kep_order, d->limiter, d->sgs, d->tile < 0 ? 0 : d->tile};

    // ---- blocks, metrics, work buffers
    c->hb.resize(d->nblocks);
    for (int b = 0; b < d->nblocks; ++b) {
        const wm_block& src = d->blocks[b];
        BlockDev& B = c->hb[b];
        B.ng = src.ng;
        for (int a = 0; a < 3; ++a) { B.n[a] = src.n[a]; B.N[a] = src.n[a] + 2 * src.ng; }
        B.case_id = 0;
        B.plane = (long long)B.N[1] * B.N[2];
        B.ncell = B.plane * B.N[0];
        for (int f = 0; f < 6; ++f) B.wall[f] = -1;
        if (B.ncell * WM_NMET >= (1LL << 31))
            return bail(fail(WM_E_UNSUPPORTED, "block %d: %lld cells exceed the 32-bit metric index range "
                             "(split the block)", b, B.ncell));
        double* met = nullptr;
        if ((r = dev_upload(c, &met, src.metrics, (size_t)WM_NMET * B.ncell))) return bail(r);
        B.met = met;
        B.met32 = nullptr;
        if (d->precision == WM_PREC_MIXED) {
            std::vector<float> m32((size_t)WM_NMET * B.ncell);
            for (size_t i = 0; i < m32.size(); ++i) m32[i] = (float)src.metrics[i];
            float* p32 = nullptr;
            if ((r = dev_upload(c, &p32, m32.data(), m32.size()))) return bail(r);
            B.met32 = p32;
        }
        for (int s = 0; s < 2; ++s) {
            double* w = nullptr;
            if ((r = dev_alloc(c, &w, 5 * (size_t)B.ncell))) return bail(r);
            CK(cudaMemset(w, 0, sizeof(double) * 5 * B.ncell));
            c->work[s].push_back(w);
        }
    }

    // ---- wall-modelled faces
    for (int w = 0; w < d->nwalls; ++w) {
        const wm_wall& src = d->walls[w];
        BlockDev& B = c->hb[src.block];
        const int ta = src.axis == 0 ? 1 : 0, tb = src.axis == 2 ? 1 : 2;
        WallDev W{};
        W.block = src.block; W.axis = src.axis; W.side = src.side; W.n_match = src.n_match;
        W.isothermal = src.isothermal; W.n_iter = src.n_iter;
        W.nt1 = B.n[ta]; W.nt2 = B.n[tb];
        W.T_wall = src.T_wall; W.kappa = src.kappa; W.B = src.B; W.ekb = std::exp(-src.kappa * src.B);
        const size_t nf = (size_t)W.nt1 * W.nt2;
        double* gm = nullptr;
        if ((r = dev_upload(c, &gm, src.geom, 5 * nf))) return bail(r);
        W.geom = gm;
        if ((r = dev_alloc(c, &W.F, 5 * nf))) return bail(r);
        if ((r = dev_alloc(c, &W.tq, 2 * nf))) return bail(r);
        c->max_wall_faces = std::max(c->max_wall_faces, (int)nf);
        if (B.wall[2 * src.axis + src.side] >= 0) return bail(fail(WM_E_INVALID, "two walls on one face"));
        B.wall[2 * src.axis + src.side] = w;
        c->hw.push_back(W);
    }
    if ((r = dev_upload(c, &c->d_walls, c->hw.data(), c->hw.size()))) return bail(r);

    // ---- ghost programs and BC constants
    if ((r = dev_upload(c, &c->d_bc, d->bc_table, 8 * (size_t)std::max(d->nbc, 1)))) return bail(r);
    if ((r = upload_prog(c, &c->prog_rhs, d->ghost_rhs))) return bail(r);
    if ((r = upload_prog(c, &c->prog_all, d->ghost_all))) return bail(r);
    if ((r = dev_alloc(c, &c->stash, 5 * (size_t)std::max(d->ghost_all.count, 1)))) return bail(r);

    // ---- synthetic inflow
    if (d->inflow) {
        const wm_inflow& I = *d->inflow;
        if (I.block < 0 || I.block >= d->nblocks) return bail(fail(WM_E_INVALID, "inflow block"));
        c->has_inflow = true;
        c->inflow = I;
        c->inflow_block = I.block;
        if ((r = dev_upload(c, &c->d_modes, I.modes, 12 * (size_t)I.n_modes))) return bail(r);
        if ((r = dev_upload(c, &c->d_table, I.table, 7 * (size_t)I.n_tab))) return bail(r);
        const BlockDev& B = c->hb[I.block];
        c->inflow_n = (long long)B.ng * B.plane;
        if ((r = dev_alloc(c, &c->inflow_buf, 5 * (size_t)c->inflow_n))) return bail(r);
    }

    // ---- sponge means
    if (d->sponge.enabled) {
        c->sponge = true;
        for (int b = 0; b < d->nblocks; ++b) {
            const BlockDev& B = c->hb[b];
            double* m = nullptr;
            if ((r = dev_alloc(c, &m, 5 * (size_t)B.N[0] * B.N[1]))) return bail(r);
            c->spmean.push_back(m);
            c->sponge_rows = std::max(c->sponge_rows, B.n[0] * B.n[1]);
        }
    }

    // ---- tiles, reduction scratch
    int tj, tk;
    tile_shape(c->opts.tile, &tj, &tk);
    build_tiles(c, tj, tk, choose_chunk(c, tj, tk, d->chunk));
    if ((r = dev_upload(c, &c->d_tiles, c->tiles.data(), c->tiles.size()))) return bail(r);
    if ((r = dev_alloc(c, &c->d_cmf_part, c->tiles.size()))) return bail(r);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    long long maxcells = 0;
    for (const BlockDev& B : c->hb) maxcells = std::max(maxcells, (long long)B.n[0] * B.n[1] * B.n[2]);
    (void)sms;
    c->dt_ctas = (int)std::max(1LL, (maxcells + 255) / 256);      // one interior cell per thread
    if ((r = dev_alloc(c, &c->d_dt_part, (size_t)c->dt_ctas * d->nblocks))) return bail(r);
    if ((r = dev_alloc(c, &c->d_counter, 2))) return bail(r);
    CK(cudaMemset(c->d_counter, 0, 2 * sizeof(unsigned)));
    if ((r = dev_alloc(c, &c->d_cmf_delta, 1))) return bail(r);
    CK(cudaMemset(c->d_cmf_delta, 0, sizeof(double)));
    if ((r = dev_alloc(c, &c->d_dt_tmp, 1))) return bail(r);

    if ((r = dev_upload(c, &c->d_case, &c->hc, 1))) return bail(r);
    if ((r = dev_upload(c, &c->d_blocks, c->hb.data(), c->hb.size()))) return bail(r);
    CK(cudaDeviceSynchronize());
    *out = c;
    return WM_OK;
}

int wm_apply_bcs(wm_case* c, double* const* q, double time, void* stream) {
    if (!c || !q) return fail(WM_E_INVALID, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    int r;
    if ((r = fill_inflow(c, time, 0.0, nullptr, s))) return r;
    LaunchScope ls(c, WM_KIND_GHOST, s, c->prog_all.count ? 2 : 0);
    CK(launch_ghost(ghost_args(c, c->prog_all, q, true), s));
    return WM_OK;
}

int wm_rhs(wm_case* c, double* const* q, double* const* rr, double time, void* stream) {
    if (!c || !q || !rr) return fail(WM_E_INVALID, "null argument");
    return run_stage(c, 0, q, nullptr, rr, nullptr, time, 0.0, (cudaStream_t)stream);
}

int wm_max_dt(wm_case* c, const double* const* q, double* dt_dev, void* stream) {
    if (!c || !q || !dt_dev) return fail(WM_E_INVALID, "null argument");
    return run_dt(c, const_cast<double* const*>(q), false, true, dt_dev, (cudaStream_t)stream);
}

int wm_advance(wm_case* c, double* const* q_in, double* const* q_out, const double* dt_dev, double time,
               void* stream) {
    if (!c || !q_in || !q_out || !dt_dev) return fail(WM_E_INVALID, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    int r;
    double* const* w0 = c->work[0].data();
    double* const* w1 = c->work[1].data();
    if ((r = run_stage(c, 1, q_in, q_in, w0, dt_dev, time, 0.0, s))) return r;
    if ((r = run_stage(c, 2, w0, q_in, w1, dt_dev, time, 1.0, s))) return r;
    if ((r = run_stage(c, 3, w1, q_in, q_out, dt_dev, time, 0.5, s))) return r;
    if (c->hc.cmf_dir >= 0 && (r = run_dt(c, q_out, true, false, nullptr, s))) return r;
    return WM_OK;
}

int wm_step(wm_case* c, double* const* q_in, double* const* q_out, double* dt_dev, double time, void* stream) {
    int r = wm_max_dt(c, q_in, dt_dev, stream);
    if (r) return r;
    return wm_advance(c, q_in, q_out, dt_dev, time, stream);
}

int wm_step_fused(wm_case* c, double* const* q_in, double* const* q_out, const double* dt_in, double* dt_next,
                  double time, void* stream) {
    if (!c || !q_in || !q_out || !dt_in || !dt_next) return fail(WM_E_INVALID, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    int r;
    double* const* w0 = c->work[0].data();
    double* const* w1 = c->work[1].data();
    if ((r = run_stage(c, 1, q_in, q_in, w0, dt_in, time, 0.0, s))) return r;
    if ((r = run_stage(c, 2, w0, q_in, w1, dt_in, time, 1.0, s))) return r;
    if ((r = run_stage(c, 3, w1, q_in, q_out, dt_in, time, 0.5, s))) return r;
    return run_dt(c, q_out, c->hc.cmf_dir >= 0, true, dt_next, s);
}

int wm_wall_stats(wm_case* c, const double* const* q, double* const* out, void* stream) {
    if (!c || !q || !out) return fail(WM_E_INVALID, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    if (c->hw.empty()) return WM_OK;
    WallArgs W{};
    W.blocks = c->d_blocks; W.cases = c->d_case; W.walls = c->d_walls;
    W.nwalls = (int)c->hw.size(); W.max_faces = c->max_wall_faces;
    W.Pr13 = c->Pr13; W.Pr3 = c->Pr3; W.kader_beta = c->kader_beta;
    for (int b = 0; b < c->nblocks; ++b) W.q[b] = q[b];
    {
        LaunchScope ls(c, WM_KIND_WALL, s);
        CK(launch_wall(W, s));
    }
    for (size_t w = 0; w < c->hw.size(); ++w) {
        const size_t nf = (size_t)c->hw[w].nt1 * c->hw[w].nt2;
        CK(cudaMemcpyAsync(out[w], c->hw[w].tq, sizeof(double) * 2 * nf, cudaMemcpyDeviceToDevice, s));
    }
    return WM_OK;
}

int wm_profile_enable(wm_case* c, int enable) {
    if (!c) return fail(WM_E_INVALID, "null case");
    for (auto& r : c->recs) { c->pool.push_back(r.a); c->pool.push_back(r.b); }
    c->recs.clear();
    for (int k = 0; k < WM_NKINDS; ++k) c->nlaunch[k] = 0;
    c->prof = enable != 0;
    return WM_OK;
}

int wm_profile_read(wm_case* c, int kind, double* ms_total, long long* launches) {
    if (!c || kind < -1 || kind >= WM_NKINDS) return fail(WM_E_INVALID, "bad profile query");
    double ms = 0.0;
    for (auto& r : c->recs) {
        if (kind >= 0 && r.kind != kind) continue;
        CK(cudaEventSynchronize(r.b));
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, r.a, r.b));
        ms += t;
    }
    long long n = 0;
    for (int k = 0; k < WM_NKINDS; ++k)
        if (kind < 0 || k == kind) n += c->nlaunch[k];
    if (ms_total) *ms_total = ms;
    if (launches) *launches = n;
    return WM_OK;
}

}  // extern "C"
