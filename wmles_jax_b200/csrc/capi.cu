// C ABI of libwmles_cuda.so (include/wmles_cuda.h): case set-up and step orchestration.
//
// A wm_case owns one case's device data (metrics, ghost programs, wall geometry, work
// states, inflow/sponge buffers).  Launches run on a View: the concatenated device tables
// (blocks, per-case constants, wall faces, stage tiles, ghost-program segments) and the
// reduction scratch of a set of cases.  Every wm_case carries a View of itself for the
// single-case entry points; a wm_batch is a View over several resident cases, so one
// launch per kernel and stage advances all of them.  The stage work list is cut for the
// whole view (longer chunks along i when many cases share the GPU).  Per-case reductions
// (CFL minimum; constant-mass-flux sum over fixed per-column, per-plane partials)
// run in a fixed order, so a case's result depends neither on the chunk length nor on what
// else is in the batch.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "wm_internal.cuh"
#include "stage.cuh"
#include "aux.cuh"
#include "stats.cuh"
#include "derived.cuh"
#include "geom.cuh"

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

// launch accounting / event timing (wm_profile_*)
struct Prof {
    long long nlaunch[WM_NKINDS] = {0, 0, 0, 0, 0};
    bool on = false;
    struct Rec { int kind; cudaEvent_t a, b; };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;

    cudaEvent_t event() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void reset(bool enable) {
        for (auto& r : recs) { pool.push_back(r.a); pool.push_back(r.b); }
        recs.clear();
        for (int k = 0; k < WM_NKINDS; ++k) nlaunch[k] = 0;
        on = enable;
    }
    ~Prof() {
        for (auto& r : recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
    }
};

// brackets one launch of `kind`: counts it and, when profiling, records an event pair
struct LaunchScope {
    Prof* p;
    int slot = -1;
    cudaStream_t s;
    LaunchScope(Prof* p_, int kind, cudaStream_t s_, int n = 1) : p(p_), s(s_) {
        p->nlaunch[kind] += n;
        if (p->on && n > 0) {
            Prof::Rec r{kind, p->event(), p->event()};
            cudaEventRecord(r.a, s);
            p->recs.push_back(r);
            slot = (int)p->recs.size() - 1;
        }
    }
    ~LaunchScope() {
        if (slot >= 0) cudaEventRecord(p->recs[slot].b, s);
    }
};

struct Owner {
    std::vector<void*> allocs;
    ~Owner() {
        for (void* p : allocs) cudaFree(p);
    }
    template <typename T>
    int alloc(T** p, size_t count) {
        void* v = nullptr;
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(&v, sizeof(T) * count);
        if (e != cudaSuccess) return fail(WM_E_CUDA, "cudaMalloc(%zu bytes): %s", sizeof(T) * count, cudaGetErrorString(e));
        allocs.push_back(v);
        *p = static_cast<T*>(v);
        return WM_OK;
    }
    template <typename T>
    int upload(T** p, const T* host, size_t count) {
        int r = alloc(p, count);
        if (r) return r;
        if (count && host) CK(cudaMemcpy(*p, host, sizeof(T) * count, cudaMemcpyHostToDevice));
        return WM_OK;
    }
};

struct View;

}  // namespace

namespace wm {
int set_error(int code, const char* msg) {
    g_err = msg;
    return code;
}
}  // namespace wm

struct wm_case {
    int device = 0;
    Owner mem;
    // host copies of the case-local descriptors (block / wall indices local to the case)
    std::vector<BlockDev> hb;
    CaseDev hc{};
    std::vector<WallDev> hw;
    int chunk_req = 0;                   // planes per stage-kernel CTA requested (0: automatic)
    StageOpts opts{};
    std::vector<double*> work[2];
    GhostProg prog_rhs, prog_all;
    double* stash = nullptr;
    double* d_bc = nullptr;
    bool has_inflow = false;
    int inflow_block = -1;
    double *d_modes = nullptr, *d_table = nullptr, *inflow_buf = nullptr, *inflow_raw = nullptr;
    double* inflow_prof = nullptr;       // 6 x inflow_n time-independent profile factors
    double* inflow_cz = nullptr;         // extruded inflow plane: cos / sin (kz z) tables (else null)
    BlockDev* d_inflow_block = nullptr;  // the inflow block's descriptor, for the set-up kernels
    wm_inflow inflow{};
    long long inflow_n = 0;
    std::vector<double*> spmean;         // per block, null without sponge
    std::vector<int> sp_rows;            // (block, interior row) pairs of the rows that reach into the sponge
    double* ps_part = nullptr;           // plane-statistics scratch (PS_NQ x max Nj x PS_CHUNKS)
    unsigned* ps_counter = nullptr;
    View* self = nullptr;                // the case as a view of one case
    unsigned* d_status = nullptr;        // status word (WM_ST_* bits)
    Prof prof;
    ~wm_case();
};

namespace {

struct View {
    Owner mem;
    std::vector<wm_case*> members;
    int nblocks = 0, ncases = 0;
    std::vector<BlockDev> hb;
    std::vector<CaseDev> hc;
    std::vector<WallDev> hw;
    std::vector<Tile> tiles;             // stage work list: (j,k) columns of every block, cut along i
    std::vector<int> cta_first;          // balanced split: CTA c runs tiles [cta_first[c], cta_first[c+1])
                                         // (empty: one tile per CTA)
    int* d_cta_first = nullptr;
    std::vector<int> case_block_start;
    std::vector<int> cmf_slot_start, case_slot_start;   // constant-mass-flux partial slots
    std::vector<GhostSeg> seg_rhs, seg_all;
    int total_rhs = 0, total_all = 0;
    BlockDev* d_blocks = nullptr;
    CaseDev* d_cases = nullptr;
    WallDev* d_walls = nullptr;
    Tile* d_tiles = nullptr;
    int* d_case_slot_start = nullptr;
    GhostSeg *d_seg_rhs = nullptr, *d_seg_all = nullptr;
    double *cmf_part = nullptr, *cmf_delta = nullptr;
    unsigned long long* dt_key = nullptr;   // CFL pass: per-case minimum keys
    unsigned* counters = nullptr;        // [0]: CFL reduction, [1]: constant-mass-flux reduction
    std::vector<int> cta_start;          // CFL pass: first CTA of each view block (+ total)
    std::vector<int> gcta_start;         // same for the blocks' ghost cells (output ghost fill)
    int max_wall_faces = 0;
    std::vector<int> sp_rows;            // (view block, row) pairs of the sponge rows of every case
    int* d_sp_rows = nullptr;
    bool any_sponge = false, any_cmf = false;
    StageOpts opts{};
};

int upload_prog(wm_case* c, GhostProg* g, const wm_ghost_program& p) {
    g->count = p.count;
    int r;
    if ((r = c->mem.upload(&g->dst, p.dst, 2 * (size_t)p.count))) return r;
    if ((r = c->mem.upload(&g->src, p.src, 2 * (size_t)p.count))) return r;
    if ((r = c->mem.upload(&g->ops, p.ops, 2 * (size_t)p.count))) return r;
    if ((r = c->mem.upload(&g->op_code, p.op_code, (size_t)p.nops))) return r;
    if ((r = c->mem.upload(&g->op_nrm, p.op_nrm, 3 * (size_t)p.nops))) return r;
    return WM_OK;
}

// every index of a ghost-cell program inside its arrays: the gather kernel trusts them
int validate_program(const wm_case_desc* d, const wm_ghost_program& p, const char* name) {
    if (p.count < 0 || p.nops < 0) return fail(WM_E_INVALID, "%s: negative count", name);
    if (p.count > 0 && (!p.dst || !p.src || !p.ops)) return fail(WM_E_INVALID, "%s: null arrays", name);
    if (p.nops > 0 && (!p.op_code || !p.op_nrm)) return fail(WM_E_INVALID, "%s: null op arrays", name);
    auto cells = [&](int b) {
        const wm_block& B = d->blocks[b];
        return (long long)(B.n[0] + 2 * B.ng) * (B.n[1] + 2 * B.ng) * (B.n[2] + 2 * B.ng);
    };
    long long inflow_n = 0;
    if (d->inflow) {
        const wm_block& B = d->blocks[d->inflow->block];
        inflow_n = (long long)B.ng * (B.n[1] + 2 * B.ng) * (B.n[2] + 2 * B.ng);
    }
    for (int e = 0; e < p.count; ++e) {
        const int db = p.dst[2 * e], dc = p.dst[2 * e + 1];
        if (db < 0 || db >= d->nblocks || dc < 0 || dc >= cells(db))
            return fail(WM_E_INVALID, "%s entry %d: destination out of range", name, e);
        const int kind = p.src[2 * e] >> 24, sb = p.src[2 * e] & 0xffffff, sc = p.src[2 * e + 1];
        const bool ok = kind == WM_SRC_CELL ? (sb < d->nblocks && sc >= 0 && sc < cells(sb))
                        : kind == WM_SRC_INFLOW ? (d->inflow && sc >= 0 && sc < inflow_n)
                        : kind == WM_SRC_CONST ? (sb < d->nbc) : false;
        if (!ok) return fail(WM_E_INVALID, "%s entry %d: source out of range", name, e);
        const int o0 = p.ops[2 * e], no = p.ops[2 * e + 1];
        if (o0 < 0 || no < 0 || (long long)o0 + no > p.nops)
            return fail(WM_E_INVALID, "%s entry %d: map chain out of range", name, e);
    }
    for (int o = 0; o < p.nops; ++o) {
        const int code = p.op_code[o] & 0xff, bc = (p.op_code[o] >> 8) & 0xff;
        if (code < WM_OP_SLIP || code > WM_OP_FARFIELD || ((code != WM_OP_SLIP) && bc >= d->nbc))
            return fail(WM_E_INVALID, "%s map %d: bad code or BC id", name, o);
    }
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
        if (B.ng != 3) return fail(WM_E_UNSUPPORTED, "block %d: ng=%d (this library supports ng=3)", b, B.ng);
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
    if (d->cmf_dir > 2) return fail(WM_E_INVALID, "cmf_dir=%d", d->cmf_dir);
    if (!(d->cfl > 0)) return fail(WM_E_INVALID, "cfl must be positive");
    for (int w = 0; w < d->nwalls; ++w) {
        const wm_wall& W = d->walls[w];
        if (!W.geom) return fail(WM_E_INVALID, "wall %d: null geometry", w);
        if (W.n_iter < 0 || W.n_iter > 1000) return fail(WM_E_INVALID, "wall %d: n_iter=%d", w, W.n_iter);
    }
    if (d->nbc < 0 || (d->nbc > 0 && !d->bc_table)) return fail(WM_E_INVALID, "bad BC table");
    if (d->inflow) {
        const wm_inflow& I = *d->inflow;
        if (I.block < 0 || I.block >= d->nblocks) return fail(WM_E_INVALID, "inflow block %d", I.block);
        if (I.n_modes < 1 || I.n_tab < 2 || !I.modes || !I.table) return fail(WM_E_INVALID, "bad inflow tables");
        if (!(I.L > 0)) return fail(WM_E_INVALID, "inflow length scale must be positive");
        const int Nk = d->blocks[I.block].n[2] + 2 * d->blocks[I.block].ng;
        if (Nk > IN_ROW_MAX_NK)
            return fail(WM_E_UNSUPPORTED, "inflow block: %d cells along k with ghosts, above %d", Nk, IN_ROW_MAX_NK);
    }
    if (d->sponge.enabled && !(d->sponge.x_end_l > d->sponge.x_start_l && d->sponge.L > 0))
        return fail(WM_E_INVALID, "bad sponge extent");
    int r;
    if ((r = validate_program(d, d->ghost_rhs, "ghost_rhs"))) return r;
    if ((r = validate_program(d, d->ghost_all, "ghost_all"))) return r;
    return WM_OK;
}

// planes per stage-kernel CTA: wave quantisation against the chunk prologue cost
int choose_chunk(const std::vector<BlockDev>& hb, const StageOpts& opts, int tj, int tk, int requested) {
    if (requested > 0) return requested;
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int occ = stage_ctas_per_sm(opts);
    if (occ < 1) occ = 1;
    const long long slots = (long long)sms * occ;
    int nimax = 0;
    for (const BlockDev& B : hb) nimax = std::max(nimax, B.n[0]);
    double best = 1e300;
    int best_ic = nimax;
    for (int ic = 4; ic <= std::max(4, nimax); ++ic) {
        long long ctas = 0;
        for (const BlockDev& B : hb) {
            const long long jk = (long long)((B.n[1] + tj - 1) / tj) * ((B.n[2] + tk - 1) / tk);
            ctas += jk * ((B.n[0] + ic - 1) / ic);
        }
        const long long waves = (ctas + slots - 1) / slots;
        const double cost = double(waves) * (std::min(ic, nimax) + 3);
        if (cost < best - 1e-9) { best = cost; best_ic = ic; }
    }
    return best_ic;
}

// resident stage-kernel CTAs of the whole GPU
int stage_slots(const StageOpts& opts) {
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int occ = stage_ctas_per_sm(opts);
    return sms * (occ < 1 ? 1 : occ);
}

// wave split, for views with fewer (j,k) columns than resident CTAs and one plane count n0:
// every column is cut at the same planes into q = slots / C equal chunks over [0, n0 - x)
// (q full waves, all columns in lockstep, so halo reads of neighbouring columns hit L2), and
// the last x planes of every column go to the r = slots - q C CTAs left over, each taking
// the tail of columns m, m + r, m + 2 r, ... in turn (again in lockstep).  x balances the
// chunk length against the tail CTAs' segments; each segment costs `prologue` planes more.
// Returns the slowest CTA's cost in planes (1e300 when the split does not apply).
double build_waves(View* v, int tj, int tk, int slots, double prologue) {
    struct Col { int b, j0, k0; };
    std::vector<Col> cols;
    const int n0 = v->hb[0].n[0];
    for (int b = 0; b < v->nblocks; ++b) {
        const BlockDev& B = v->hb[b];
        if (B.n[0] != n0) return 1e300;
        for (int j0 = B.ng; j0 < B.ng + B.n[1]; j0 += tj)
            for (int k0 = B.ng; k0 < B.ng + B.n[2]; k0 += tk) cols.push_back(Col{b, j0, k0});
    }
    const int C = (int)cols.size();
    const int q = slots / C, r = slots - q * C;
    if (q < 1 || r < 1) return 1e300;
    const int m = (C + r - 1) / r;                 // tail segments of the busiest tail CTA
    double best = 1e300;
    int bx = 0;
    for (int x = 16; x < n0 / 2; ++x) {           // tail segments of at least 16 planes
        const double main_cost = std::ceil(double(n0 - x) / q) + prologue;
        const double tail_cost = m * (x + prologue);
        const double cost = std::max(main_cost, tail_cost);
        if (cost < best - 1e-9) { best = cost; bx = x; }
    }
    if (bx == 0) return 1e300;
    const int L = (n0 - bx + q - 1) / q;
    v->tiles.clear();
    v->cta_first.assign(1, 0);
    for (int w = 0; w < q; ++w)
        for (const Col& c : cols) {
            const int ng = v->hb[c.b].ng;
            const int lo = w * L, hi = std::min((w + 1) * L, n0 - bx);
            if (hi > lo) v->tiles.push_back(Tile{c.b, c.j0, c.k0, ng + lo, ng + hi});
            v->cta_first.push_back((int)v->tiles.size());
        }
    for (int t = 0; t < r; ++t) {
        for (int c = t; c < C; c += r) {
            const int ng = v->hb[cols[c].b].ng;
            v->tiles.push_back(Tile{cols[c].b, cols[c].j0, cols[c].k0, ng + n0 - bx, ng + n0});
        }
        v->cta_first.push_back((int)v->tiles.size());
    }
    return best;
}

// constant-mass-flux partial slots of a view: one per (column, interior plane) of each block,
// independent of how the columns are cut into CTAs
void cmf_slots(View* v, int tj, int tk) {
    v->cmf_slot_start.assign(1, 0);
    for (int b = 0; b < v->nblocks; ++b) {
        const BlockDev& B = v->hb[b];
        const int cols = ((B.n[1] + tj - 1) / tj) * ((B.n[2] + tk - 1) / tk);
        v->cmf_slot_start.push_back(v->cmf_slot_start.back() + cols * B.n[0]);
    }
    v->case_slot_start.clear();
    for (int c = 0; c <= v->ncases; ++c) v->case_slot_start.push_back(v->cmf_slot_start[v->case_block_start[c]]);
}

// chunked split: every column cut into chunks of ic planes, one chunk per CTA
void build_tiles(View* v, int tj, int tk, int ic) {
    v->tiles.clear();
    v->cta_first.clear();
    for (int b = 0; b < v->nblocks; ++b) {
        const BlockDev& B = v->hb[b];
        const int ng = B.ng;
        for (int i0 = ng; i0 < ng + B.n[0]; i0 += ic)
            for (int j0 = ng; j0 < ng + B.n[1]; j0 += tj)
                for (int k0 = ng; k0 < ng + B.n[2]; k0 += tk)
                    v->tiles.push_back(Tile{b, j0, k0, i0, std::min(i0 + ic, ng + B.n[0])});
    }
}

bool same_opts(const StageOpts& a, const StageOpts& b) {
    return a.precision == b.precision && a.scheme == b.scheme && a.kep_order == b.kep_order &&
           a.limiter == b.limiter && a.sgs == b.sgs && a.tile == b.tile;
}

GhostSeg segment(const wm_case* c, const GhostProg& p, int start, int block0) {
    GhostSeg g{};
    g.dst = p.dst; g.src = p.src; g.ops = p.ops; g.op_code = p.op_code; g.op_nrm = p.op_nrm;
    g.bc = c->d_bc;
    g.inflow = c->inflow_buf;
    g.inflow_n = c->inflow_n;
    g.start = start; g.count = p.count; g.block0 = block0;
    g.gamma = c->hc.gamma; g.gm1 = c->hc.gm1; g.Rg = c->hc.Rg;
    return g;
}

// concatenated device tables and reduction scratch of `cases`
int build_view(View* v, wm_case* const* cases, int n) {
    if (n < 1 || n > MAX_CASES) return fail(WM_E_INVALID, "a view holds 1..%d cases, got %d", MAX_CASES, n);
    for (int ci = 0; ci < n; ++ci) {
        wm_case* c = cases[ci];
        if (!c) return fail(WM_E_INVALID, "null case %d", ci);
        if (ci > 0 && !same_opts(c->opts, cases[0]->opts))
            return fail(WM_E_UNSUPPORTED, "cases of one batch must share precision, scheme, SGS model and tile shape");
        const int bo = (int)v->hb.size(), wo = (int)v->hw.size();
        if (bo + (int)c->hb.size() > WM_MAX_BLOCKS)
            return fail(WM_E_UNSUPPORTED, "a batch holds at most %d blocks", WM_MAX_BLOCKS);
        v->members.push_back(c);
        v->case_block_start.push_back(bo);
        for (BlockDev B : c->hb) {
            B.case_id = ci;
            for (int f = 0; f < 6; ++f)
                if (B.wall[f] >= 0) B.wall[f] += wo;
            v->hb.push_back(B);
        }
        for (WallDev W : c->hw) {
            W.block += bo;
            v->max_wall_faces = std::max(v->max_wall_faces, W.nt1 * W.nt2);
            v->hw.push_back(W);
        }
        v->hc.push_back(c->hc);
        v->seg_rhs.push_back(segment(c, c->prog_rhs, v->total_rhs, bo));
        v->total_rhs += c->prog_rhs.count;
        v->seg_all.push_back(segment(c, c->prog_all, v->total_all, bo));
        v->total_all += c->prog_all.count;
        for (size_t p = 0; p < c->sp_rows.size(); p += 2) {
            v->sp_rows.push_back(bo + c->sp_rows[p]);
            v->sp_rows.push_back(c->sp_rows[p + 1]);
        }
        v->any_sponge = v->any_sponge || c->hc.sponge;
        v->any_cmf = v->any_cmf || c->hc.cmf_dir >= 0;
    }
    v->case_block_start.push_back((int)v->hb.size());
    v->nblocks = (int)v->hb.size();
    v->ncases = n;
    v->opts = cases[0]->opts;
    // the chunk length is chosen for the whole set (results do not depend on it)
    int req = cases[0]->chunk_req;
    for (int ci = 1; ci < n; ++ci)
        if (cases[ci]->chunk_req != req) req = 0;
    int tj, tk;
    tile_shape(v->opts.tile, &tj, &tk);
    const int ic = choose_chunk(v->hb, v->opts, tj, tk, req);
    build_tiles(v, tj, tk, ic);
    if (req == 0) {
        // automatic: the wave split when its slowest CTA costs less than the chunked grid's
        // waves
        const int slots = stage_slots(v->opts);
        const long long nt = (long long)v->tiles.size();
        // a segment's prologue (four planes staged and converted, two gradient planes, one
        // face plane, with little overlap) charged as 6 planes in this comparison
        const double chunked = double((nt + slots - 1) / slots) * (ic + 6);
        View trial;
        trial.hb = v->hb; trial.nblocks = v->nblocks;
        if (build_waves(&trial, tj, tk, slots, 6.0) < chunked) {
            v->tiles = trial.tiles;
            v->cta_first = trial.cta_first;
        }
    }
    cmf_slots(v, tj, tk);
    v->cta_start.assign(1, 0);                  // one interior cell per thread of the CFL pass
    v->gcta_start.assign(1, 0);                 // one ghost cell per thread
    for (const BlockDev& B : v->hb) {
        v->cta_start.push_back(v->cta_start.back() + (int)(((long long)B.n[0] * B.n[1] * B.n[2] + DT_NT - 1) / DT_NT));
        v->gcta_start.push_back(v->gcta_start.back() + (int)((ghost_cells(B) + DT_NT - 1) / DT_NT));
    }
    int r;
    Owner& m = v->mem;
    if ((r = m.upload(&v->d_blocks, v->hb.data(), v->hb.size()))) return r;
    if ((r = m.upload(&v->d_cases, v->hc.data(), v->hc.size()))) return r;
    if ((r = m.upload(&v->d_walls, v->hw.data(), v->hw.size()))) return r;
    if ((r = m.upload(&v->d_tiles, v->tiles.data(), v->tiles.size()))) return r;
    if (!v->cta_first.empty())
        if ((r = m.upload(&v->d_cta_first, v->cta_first.data(), v->cta_first.size()))) return r;
    if ((r = m.upload(&v->d_case_slot_start, v->case_slot_start.data(), v->case_slot_start.size()))) return r;
    if ((r = m.upload(&v->d_seg_rhs, v->seg_rhs.data(), v->seg_rhs.size()))) return r;
    if ((r = m.upload(&v->d_seg_all, v->seg_all.data(), v->seg_all.size()))) return r;
    if (!v->sp_rows.empty())
        if ((r = m.upload(&v->d_sp_rows, v->sp_rows.data(), v->sp_rows.size()))) return r;
    if ((r = m.alloc(&v->cmf_part, (size_t)v->cmf_slot_start.back()))) return r;
    if ((r = m.alloc(&v->cmf_delta, (size_t)n))) return r;
    CK(cudaMemset(v->cmf_delta, 0, sizeof(double) * n));
    {
        const std::vector<unsigned long long> empty((size_t)n, DT_KEY_EMPTY);
        if ((r = m.upload(&v->dt_key, empty.data(), empty.size()))) return r;
    }
    if ((r = m.alloc(&v->counters, 2))) return r;
    CK(cudaMemset(v->counters, 0, 2 * sizeof(unsigned)));
    return WM_OK;
}

int fill_inflow(View* v, Prof* pf, const double* times, double time_dt, const double* const* dt, cudaStream_t s) {
    for (int ci = 0; ci < v->ncases; ++ci) {
        wm_case* c = v->members[ci];
        if (!c->has_inflow) continue;
        const int vb = v->case_block_start[ci] + c->inflow_block;
        const BlockDev& B = v->hb[vb];
        InflowArgs I{};
        I.block = v->d_blocks + vb;
        I.modes = c->d_modes; I.table = c->d_table;
        I.n_modes = c->inflow.n_modes; I.n_tab = c->inflow.n_tab;
        I.U_inf = c->inflow.U_inf; I.L = c->inflow.L; I.rho_inf = c->inflow.rho_inf; I.p_inf = c->inflow.p_inf;
        I.gm1 = c->hc.gm1;
        I.time0 = times[ci]; I.time_dt = time_dt; I.dt = dt ? dt[ci] : nullptr;
        I.raw = c->inflow_raw;
        I.out = c->inflow_buf;
        I.prof = c->inflow_prof;
        I.cz = c->inflow_cz;
        LaunchScope ls(pf, WM_KIND_SOURCE, s, IN_LAUNCHES);
        CK(launch_inflow(I, B.N[1], B.N[2], B.ng, s));
    }
    return WM_OK;
}

// one RHS evaluation fused with RK stage `stage` (0 = plain RHS) for every case of the view;
// state pointers per view block, time steps and times per case
int run_stage(View* v, Prof* pf, int stage, double* const* q_in, const double* const* q0, double* const* q_out,
              const double* const* dt, const double* times, double time_dt, cudaStream_t s) {
    int r;
    if ((r = fill_inflow(v, pf, times, time_dt, dt, s))) return r;
    // ghost cells the RHS reads, wall-model flux overrides and sponge means: one launch
    SurfaceArgs U{};
    U.G.segs = v->d_seg_rhs; U.G.nseg = v->ncases; U.G.total = v->total_rhs; U.G.stash = nullptr;
    for (int b = 0; b < v->nblocks; ++b) { U.G.q[b] = q_in[b]; U.G.ncell[b] = v->hb[b].ncell; }
    U.W.blocks = v->d_blocks; U.W.cases = v->d_cases; U.W.walls = v->d_walls;
    U.W.nwalls = (int)v->hw.size(); U.W.max_faces = v->max_wall_faces;
    for (int b = 0; b < v->nblocks; ++b) U.W.q[b] = q_in[b];
    std::vector<const double*> spm(v->nblocks, nullptr);
    if (v->any_sponge) {
        U.S.blocks = v->d_blocks; U.S.cases = v->d_cases; U.S.nblocks = v->nblocks;
        U.S.nrows = (int)v->sp_rows.size() / 2; U.S.rows = v->d_sp_rows;
        for (int ci = 0; ci < v->ncases; ++ci)
            for (size_t b = 0; b < v->members[ci]->hb.size(); ++b) {
                const int vb = v->case_block_start[ci] + (int)b;
                U.S.q[vb] = q_in[vb];
                U.S.mean[vb] = v->members[ci]->spmean[b];
                spm[vb] = U.S.mean[vb];
            }
    }
    {
        const bool any = U.G.total > 0 || !v->hw.empty() || v->any_sponge;
        LaunchScope ls(pf, WM_KIND_GHOST, s, any ? 1 : 0);
        CK(launch_surface(U, s));
    }
    StageArgs A{};
    A.blocks = v->d_blocks; A.cases = v->d_cases; A.walls = v->d_walls;
    A.tiles = v->d_tiles; A.ntiles = (int)v->tiles.size();
    A.cta_first = v->cta_first.empty() ? nullptr : v->d_cta_first;
    A.nctas = v->cta_first.empty() ? A.ntiles : (int)v->cta_first.size() - 1;
    A.stage = stage;
    A.ncases = v->ncases;
    A.case_slot_start = v->d_case_slot_start;
    A.cmf_part = (stage == 3 && v->any_cmf) ? v->cmf_part : nullptr;
    A.cmf_counter = v->counters + 1;
    A.cmf_delta = v->cmf_delta;
    for (int ci = 0; ci < v->ncases; ++ci) A.dt[ci] = dt ? dt[ci] : nullptr;
    for (int b = 0; b < v->nblocks; ++b) {
        A.p[b].q_in = q_in[b];
        A.p[b].q0 = q0 ? q0[b] : q_in[b];
        A.p[b].q_out = q_out[b];
        A.p[b].spmean = spm[b];
        A.cmf_slot_start[b] = v->cmf_slot_start[b];
    }
    LaunchScope ls(pf, WM_KIND_STAGE, s);
    CK(launch_stage(A, v->opts, s));
    return WM_OK;
}

// the CFL / constraint pass over q; with q_src (a step's input) it also sets the ghost
// cells of q (the step's output) from q_src's
int run_dt(View* v, Prof* pf, double* const* q, bool apply_cmf, bool want_dt, double* const* dt_out,
           const double* const* q_src, cudaStream_t s) {
    DtArgs D{};
    D.blocks = v->d_blocks; D.cases = v->d_cases; D.nblocks = v->nblocks;
    D.ncta = v->cta_start.back();
    for (int b = 0; b <= v->nblocks; ++b) D.cta_start[b] = v->cta_start[b];
    D.ngcta = q_src ? v->gcta_start.back() : 0;
    for (int b = 0; b <= v->nblocks; ++b) D.gcta_start[b] = v->gcta_start[b];
    for (int b = 0; b < v->nblocks; ++b) D.q_src[b] = q_src ? q_src[b] : nullptr;
    D.ncases = v->ncases;
    for (int ci = 0; ci <= v->ncases; ++ci) D.case_block_start[ci] = v->case_block_start[ci];
    for (int b = 0; b < v->nblocks; ++b) D.q[b] = q[b];
    D.cmf_delta = apply_cmf ? v->cmf_delta : nullptr;
    D.want_dt = want_dt ? 1 : 0;
    D.met32 = v->opts.precision == WM_PREC_MIXED ? 1 : 0;
    D.dt_key = v->dt_key; D.counter = v->counters;
    for (int ci = 0; ci < v->ncases; ++ci) D.dt_out[ci] = dt_out ? dt_out[ci] : nullptr;
    LaunchScope ls(pf, WM_KIND_DT, s);
    CK(launch_dt(D, s));
    return WM_OK;
}

// SSP-RK3 of every case of the view with work states w0/w1 (per view block), then the
// constraint pass; with want_next the pass also writes each case's next CFL time step
int run_step(View* v, Prof* pf, double* const* q_in, double* const* q_out, double* const* w0, double* const* w1,
             const double* const* dt, double* const* dt_next, const double* times, bool want_next, cudaStream_t s) {
    int r;
    if ((r = run_stage(v, pf, 1, q_in, q_in, w0, dt, times, 0.0, s))) return r;
    if ((r = run_stage(v, pf, 2, w0, q_in, w1, dt, times, 1.0, s))) return r;
    if ((r = run_stage(v, pf, 3, w1, q_in, q_out, dt, times, 0.5, s))) return r;
    // constraint, next time step and the output's ghost cells in one pass
    return run_dt(v, pf, q_out, v->any_cmf, want_next, dt_next, q_in, s);
}

}  // namespace

wm_case::~wm_case() { delete self; }

namespace {
// every per-block (or per-case) pointer of an argument array is set: a null one would
// become a device fault
int check_ptrs(const void* const* p, int n, const char* what) {
    if (!p) return fail(WM_E_INVALID, "null %s array", what);
    for (int i = 0; i < n; ++i)
        if (!p[i]) return fail(WM_E_INVALID, "null %s[%d]", what, i);
    return WM_OK;
}
}  // namespace

struct wm_batch {
    View view;
    Prof prof;
    std::vector<double*> w0, w1;     // per view block: the member cases' work states
    unsigned* d_status = nullptr;    // member cases' status words, gathered (wm_batch_status)
};

namespace {
const char* status_names(unsigned st) {
    static thread_local std::string s;
    s.clear();
    const char* names[] = {"non-finite state", "non-positive density", "non-positive pressure",
                           "non-finite or non-positive time step", "wall-model Newton not settled"};
    for (int b = 0; b < 5; ++b)
        if (st & (1u << b)) { if (!s.empty()) s += ", "; s += names[b]; }
    return s.c_str();
}
}  // namespace

extern "C" {

int wm_version(void) { return WM_ABI_VERSION; }
const char* wm_last_error(void) { return g_err.c_str(); }

void wm_case_destroy(wm_case* c) { delete c; }

int wm_case_create(const wm_case_desc* d, wm_case** out) {
    if (!out) return fail(WM_E_INVALID, "null output handle");
    *out = nullptr;
    int r = validate(d);
    if (r) return r;
    wm_case* c = new wm_case();
    auto bail = [&](int code) { delete c; return code; };
    // a failed CUDA call frees the partly built case (its allocations are owned by it)
#define CKB(call)                                                                            \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return bail(fail(WM_E_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                             __FILE__, __LINE__));                                           \
    } while (0)
    CKB(cudaGetDevice(&c->device));

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
    C.Pr13 = std::pow(g.Pr, 1.0 / 3.0);
    C.Pr3 = std::pow(g.Pr, 3.0);
    C.kader_beta = std::pow(3.85 * std::pow(g.Pr, 1.0 / 3.0) - 1.3, 2.0) + 2.12 * std::log(g.Pr);
    C.cmf_dir = d->cmf_dir; C.cmf_target = d->cmf_target; C.cmf_volume = d->cmf_volume;
    C.sponge = d->sponge.enabled;
    if (C.sponge) {
        C.sp_xs = d->sponge.x_start_l;
        C.sp_inv_dx = 1.0 / (d->sponge.x_end_l - d->sponge.x_start_l);
        C.sp_sigma0 = d->sponge.strength * d->sponge.U_inf / d->sponge.L;
        C.sp_invL = 1.0 / d->sponge.L;
    }
    // automatic tile shape: 8x32 for FP64, 16x32 for the mixed form (the fastest on every
    // measured workload but the C-grid, whose 40-cell k extent the FP64 16x16 tile fits better);
    // fixed per precision, so cases created with the default can share a batch
    const int auto_tile = d->precision == WM_PREC_MIXED ? 3 : 0;
    c->opts = StageOpts{d->precision, d->scheme, d->kep_order, d->limiter, d->sgs, d->tile < 0 ? auto_tile : d->tile};

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
        // the metric table may sit in host or device memory (wm_block_geometry's output);
        // the mixed form's FP32 copy is rounded on the device from the case's FP64 copy
        const size_t nmet = (size_t)WM_NMET * B.ncell;
        cudaPointerAttributes pa{};
        CKB(cudaPointerGetAttributes(&pa, src.metrics));
        const bool on_device = pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged;
        double* met = nullptr;
        if ((r = c->mem.alloc(&met, nmet))) return bail(r);
        CKB(cudaMemcpy(met, src.metrics, sizeof(double) * nmet,
                       on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
        B.met = met;
        B.met32 = nullptr;
        if (d->precision == WM_PREC_MIXED) {
            float* p32 = nullptr;
            if ((r = c->mem.alloc(&p32, nmet))) return bail(r);
            CKB(launch_to_f32(met, p32, (long long)nmet, 0));
            B.met32 = p32;
        }
        for (int s = 0; s < 2; ++s) {
            double* w = nullptr;
            if ((r = c->mem.alloc(&w, 5 * (size_t)B.ncell))) return bail(r);
            CKB(cudaMemset(w, 0, sizeof(double) * 5 * B.ncell));
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
        if ((r = c->mem.upload(&gm, src.geom, 5 * nf))) return bail(r);
        W.geom = gm;
        if ((r = c->mem.alloc(&W.F, 5 * nf))) return bail(r);
        if ((r = c->mem.alloc(&W.tq, 2 * nf))) return bail(r);
        if (B.wall[2 * src.axis + src.side] >= 0) return bail(fail(WM_E_INVALID, "two walls on one face"));
        B.wall[2 * src.axis + src.side] = w;
        c->hw.push_back(W);
    }

    // ---- ghost programs and BC constants
    if ((r = c->mem.upload(&c->d_bc, d->bc_table, 8 * (size_t)std::max(d->nbc, 1)))) return bail(r);
    if ((r = upload_prog(c, &c->prog_rhs, d->ghost_rhs))) return bail(r);
    if ((r = upload_prog(c, &c->prog_all, d->ghost_all))) return bail(r);
    if ((r = c->mem.alloc(&c->stash, 5 * (size_t)std::max(d->ghost_all.count, 1)))) return bail(r);

    // ---- synthetic inflow
    if (d->inflow) {
        const wm_inflow& I = *d->inflow;
        if (I.block < 0 || I.block >= d->nblocks) return bail(fail(WM_E_INVALID, "inflow block"));
        c->has_inflow = true;
        c->inflow = I;
        c->inflow_block = I.block;
        if ((r = c->mem.upload(&c->d_modes, I.modes, 12 * (size_t)I.n_modes))) return bail(r);
        if ((r = c->mem.upload(&c->d_table, I.table, 7 * (size_t)I.n_tab))) return bail(r);
        const BlockDev& B = c->hb[I.block];
        c->inflow_n = (long long)B.ng * B.plane;
        if ((r = c->mem.alloc(&c->inflow_buf, 5 * (size_t)c->inflow_n))) return bail(r);
        if ((r = c->mem.alloc(&c->inflow_raw, (size_t)IN_PARTS * 3 * c->inflow_n))) return bail(r);
        if ((r = c->mem.alloc(&c->inflow_prof, 6 * (size_t)c->inflow_n))) return bail(r);
        if ((r = c->mem.upload(&c->d_inflow_block, &B, 1))) return bail(r);
        // extruded plane: every ghost row's y constant along k, z the same function of k on
        // every row (then the mode sums factor per row and per k); one component's cos / sin
        // (kz z) table must fit the mode-sum launch's shared memory
        const size_t n = (size_t)c->inflow_n;
        std::vector<double> y(n), z(n);
        CKB(cudaMemcpy(y.data(), B.met + (size_t)WM_MET_XCY * B.ncell, sizeof(double) * n, cudaMemcpyDeviceToHost));
        CKB(cudaMemcpy(z.data(), B.met + (size_t)WM_MET_XCZ * B.ncell, sizeof(double) * n, cudaMemcpyDeviceToHost));
        const int Nk = B.N[2];
        bool extruded = inflow_ext_smem(I.n_modes, Nk) <= inflow_ext_smem_max();
        for (size_t cell = 0; cell < n && extruded; ++cell) {
            const size_t k = cell % Nk;
            extruded = y[cell] == y[cell - k] && z[cell] == z[k];
        }
        InflowArgs IA{};
        IA.block = c->d_inflow_block;
        IA.modes = c->d_modes; IA.table = c->d_table;
        IA.n_modes = I.n_modes; IA.n_tab = I.n_tab;
        IA.U_inf = I.U_inf; IA.L = I.L;
        if (extruded)
            if ((r = c->mem.alloc(&c->inflow_cz, 2 * 3 * (size_t)I.n_modes * Nk))) return bail(r);
        CKB(launch_inflow_setup(IA, B.N[1], Nk, B.ng, c->inflow_prof, c->inflow_cz, 0));
    }

    // ---- sponge means
    c->spmean.assign(d->nblocks, nullptr);
    if (d->sponge.enabled) {
        for (int b = 0; b < d->nblocks; ++b) {
            const BlockDev& B = c->hb[b];
            if ((r = c->mem.alloc(&c->spmean[b], 5 * (size_t)B.N[0] * B.N[1]))) return bail(r);
            // rows outside the sponge are never written (their mean is not needed): keep them 0
            CKB(cudaMemset(c->spmean[b], 0, sizeof(double) * 5 * B.N[0] * B.N[1]));
            const int rows = B.n[0] * B.n[1];
            unsigned char* d_flags = nullptr;
            if ((r = c->mem.alloc(&d_flags, (size_t)rows))) return bail(r);
            CKB(launch_sponge_flags(B.met + (size_t)WM_MET_XCX * B.ncell, B.plane, B.N[2], B.ng, B.n[0], B.n[1],
                                    B.n[2], C.sp_invL, C.sp_xs, C.sp_inv_dx, d_flags, 0));
            std::vector<unsigned char> flags((size_t)rows);
            CKB(cudaMemcpy(flags.data(), d_flags, (size_t)rows, cudaMemcpyDeviceToHost));
            for (int row = 0; row < rows; ++row)
                if (flags[row]) { c->sp_rows.push_back(b); c->sp_rows.push_back(row); }
        }
    }

    c->chunk_req = d->chunk > 0 ? d->chunk : 0;

    // ---- plane-statistics scratch
    int max_nj = 1;
    for (const BlockDev& B : c->hb) max_nj = std::max(max_nj, B.n[1]);
    if ((r = c->mem.alloc(&c->ps_part, (size_t)PS_NQ * max_nj * PS_CHUNKS))) return bail(r);
    if ((r = c->mem.alloc(&c->ps_counter, 1))) return bail(r);
    CKB(cudaMemset(c->ps_counter, 0, sizeof(unsigned)));

    // ---- status word (every view of the case points at it)
    if ((r = c->mem.alloc(&c->d_status, 1))) return bail(r);
    CKB(cudaMemset(c->d_status, 0, sizeof(unsigned)));
    c->hc.status = c->d_status;

    c->self = new View();
    wm_case* self_list[1] = {c};
    if ((r = build_view(c->self, self_list, 1))) return bail(r);
    CKB(cudaDeviceSynchronize());
    *out = c;
    return WM_OK;
#undef CKB
}

int wm_apply_bcs(wm_case* c, double* const* q, double time, void* stream) {
    if (!c) return fail(WM_E_INVALID, "null case");
    if (int r = check_ptrs((const void* const*)q, c->self->nblocks, "q")) return r;
    cudaStream_t s = (cudaStream_t)stream;
    View* v = c->self;
    int r;
    if ((r = fill_inflow(v, &c->prof, &time, 0.0, nullptr, s))) return r;
    GhostArgs G{};
    G.segs = v->d_seg_all; G.nseg = 1; G.total = v->total_all; G.stash = c->stash;
    for (int b = 0; b < v->nblocks; ++b) { G.q[b] = q[b]; G.ncell[b] = v->hb[b].ncell; }
    LaunchScope ls(&c->prof, WM_KIND_GHOST, s, G.total ? 2 : 0);
    CK(launch_ghost(G, s));
    return WM_OK;
}

int wm_rhs(wm_case* c, double* const* q, double* const* rr, double time, void* stream) {
    if (!c) return fail(WM_E_INVALID, "null case");
    if (int r = check_ptrs((const void* const*)q, c->self->nblocks, "q")) return r;
    if (int r = check_ptrs((const void* const*)rr, c->self->nblocks, "r")) return r;
    return run_stage(c->self, &c->prof, 0, q, nullptr, rr, nullptr, &time, 0.0, (cudaStream_t)stream);
}

int wm_max_dt(wm_case* c, const double* const* q, double* dt_dev, void* stream) {
    if (!c || !dt_dev) return fail(WM_E_INVALID, "null argument");
    if (int r = check_ptrs((const void* const*)q, c->self->nblocks, "q")) return r;
    return run_dt(c->self, &c->prof, const_cast<double* const*>(q), false, true, &dt_dev, nullptr,
                  (cudaStream_t)stream);
}

int wm_advance(wm_case* c, double* const* q_in, double* const* q_out, const double* dt_dev, double time,
               void* stream) {
    if (!c || !dt_dev) return fail(WM_E_INVALID, "null argument");
    if (int r = check_ptrs((const void* const*)q_in, c->self->nblocks, "q_in")) return r;
    if (int r = check_ptrs((const void* const*)q_out, c->self->nblocks, "q_out")) return r;
    return run_step(c->self, &c->prof, q_in, q_out, c->work[0].data(), c->work[1].data(), &dt_dev, nullptr, &time,
                    false, (cudaStream_t)stream);
}

int wm_step(wm_case* c, double* const* q_in, double* const* q_out, double* dt_dev, double time, void* stream) {
    int r = wm_max_dt(c, q_in, dt_dev, stream);
    if (r) return r;
    return wm_advance(c, q_in, q_out, dt_dev, time, stream);
}

int wm_step_fused(wm_case* c, double* const* q_in, double* const* q_out, const double* dt_in, double* dt_next,
                  double time, void* stream) {
    if (!c || !dt_in || !dt_next) return fail(WM_E_INVALID, "null argument");
    if (int r = check_ptrs((const void* const*)q_in, c->self->nblocks, "q_in")) return r;
    if (int r = check_ptrs((const void* const*)q_out, c->self->nblocks, "q_out")) return r;
    return run_step(c->self, &c->prof, q_in, q_out, c->work[0].data(), c->work[1].data(), &dt_in, &dt_next, &time,
                    true, (cudaStream_t)stream);
}

int wm_case_status(wm_case* c, unsigned* status, int clear, void* stream) {
    if (!c || !status) return fail(WM_E_INVALID, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned st = 0;
    CK(cudaMemcpyAsync(&st, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    if (clear) CK(cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), s));
    CK(cudaStreamSynchronize(s));
    *status = st;
    return WM_OK;
}

int wm_check(wm_case* c, void* stream) {
    unsigned st = 0;
    if (int r = wm_case_status(c, &st, 1, stream)) return r;
    if (st & WM_ST_FATAL) return fail(WM_E_NONFINITE, "case status 0x%x: %s", st, status_names(st));
    return WM_OK;
}

int wm_wall_stats(wm_case* c, const double* const* q, double* const* out, void* stream) {
    if (!c) return fail(WM_E_INVALID, "null case");
    if (int r = check_ptrs((const void* const*)q, c->self->nblocks, "q")) return r;
    if (int r = check_ptrs((const void* const*)out, (int)c->self->hw.size(), "out")) return r;
    cudaStream_t s = (cudaStream_t)stream;
    View* v = c->self;
    if (v->hw.empty()) return WM_OK;
    WallArgs W{};
    W.blocks = v->d_blocks; W.cases = v->d_cases; W.walls = v->d_walls;
    W.nwalls = (int)v->hw.size(); W.max_faces = v->max_wall_faces;
    for (int b = 0; b < v->nblocks; ++b) W.q[b] = q[b];
    {
        LaunchScope ls(&c->prof, WM_KIND_WALL, s);
        CK(launch_wall(W, s));
    }
    for (size_t w = 0; w < v->hw.size(); ++w) {
        const size_t nf = (size_t)v->hw[w].nt1 * v->hw[w].nt2;
        CK(cudaMemcpyAsync(out[w], v->hw[w].tq, sizeof(double) * 2 * nf, cudaMemcpyDeviceToDevice, s));
    }
    return WM_OK;
}

int wm_plane_stats(wm_case* c, int block, const double* q, double* sum, void* stream) {
    if (!c || !q || !sum) return fail(WM_E_INVALID, "null argument");
    if (block < 0 || block >= c->self->nblocks) return fail(WM_E_INVALID, "block %d out of range", block);
    PlaneStatsArgs A{};
    A.block = c->self->d_blocks + block;
    A.q = q;
    A.gm1 = c->hc.gm1;
    A.Rg = c->hc.Rg;
    A.nchunks = PS_CHUNKS;
    A.part = c->ps_part;
    A.sum = sum;
    A.counter = c->ps_counter;
    CK(launch_plane_stats(A, c->hb[block].n[1], (cudaStream_t)stream));
    return WM_OK;
}

int wm_derived_fields(wm_case* c, const double* const* q, double* const* out, void* stream) {
    if (!c) return fail(WM_E_INVALID, "null case");
    if (int r = check_ptrs((const void* const*)q, c->self->nblocks, "q")) return r;
    if (int r = check_ptrs((const void* const*)out, c->self->nblocks, "out")) return r;
    View* v = c->self;
    for (int b = 0; b < v->nblocks; ++b) {
        DerivedArgs A{};
        A.block = v->d_blocks + b;
        A.cs = v->d_cases;
        A.sgs = c->opts.sgs;
        A.q = q[b];
        A.out = out[b];
        const BlockDev& B = v->hb[b];
        CK(launch_derived(A, (long long)B.n[0] * B.n[1] * B.n[2], (cudaStream_t)stream));
    }
    return WM_OK;
}

int wm_block_geometry(const double* X, const int* N, double* vol, double* xc, double* const* S,
                      double* const* xf, double* met, void* stream) {
    if (!X || !N || !vol || !xc || !S || !xf) return fail(WM_E_INVALID, "null argument");
    GeomArgs A{};
    A.X = X;
    for (int d = 0; d < 3; ++d) {
        if (N[d] < 1) return fail(WM_E_INVALID, "N[%d] = %d: every direction needs a cell", d, N[d]);
        if (!S[d] || !xf[d]) return fail(WM_E_INVALID, "null face array of direction %d", d);
        A.N[d] = N[d];
        A.S[d] = S[d];
        A.xf[d] = xf[d];
    }
    A.vol = vol;
    A.xc = xc;
    A.met = met;
    CK(launch_geometry(A, (cudaStream_t)stream));
    return WM_OK;
}

int wm_batch_create(int ncases, wm_case* const* cases, wm_batch** out) {
    if (!out || !cases) return fail(WM_E_INVALID, "null argument");
    *out = nullptr;
    wm_batch* b = new wm_batch();
    int r = build_view(&b->view, cases, ncases);
    if (r) { delete b; return r; }
    for (int ci = 0; ci < ncases; ++ci)
        for (size_t k = 0; k < cases[ci]->hb.size(); ++k) {
            b->w0.push_back(cases[ci]->work[0][k]);
            b->w1.push_back(cases[ci]->work[1][k]);
        }
    if ((r = b->view.mem.alloc(&b->d_status, (size_t)ncases))) { delete b; return r; }
    *out = b;
    return WM_OK;
}

void wm_batch_destroy(wm_batch* b) { delete b; }

int wm_batch_status(wm_batch* b, unsigned* status, void* stream) {
    if (!b || !status) return fail(WM_E_INVALID, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    CK(launch_status_gather(b->view.d_cases, b->view.ncases, b->d_status, s));
    CK(cudaMemcpyAsync(status, b->d_status, sizeof(unsigned) * b->view.ncases, cudaMemcpyDeviceToHost, s));
    return WM_OK;
}

int wm_batch_step(wm_batch* b, double* const* q_in, double* const* q_out, const double* const* dt_in,
                  double* const* dt_next, const double* times, void* stream) {
    if (!b || !times) return fail(WM_E_INVALID, "null argument");
    const View& v = b->view;
    if (int r = check_ptrs((const void* const*)q_in, v.nblocks, "q_in")) return r;
    if (int r = check_ptrs((const void* const*)q_out, v.nblocks, "q_out")) return r;
    if (int r = check_ptrs((const void* const*)dt_in, v.ncases, "dt_in")) return r;
    if (int r = check_ptrs((const void* const*)dt_next, v.ncases, "dt_next")) return r;
    return run_step(&b->view, &b->prof, q_in, q_out, b->w0.data(), b->w1.data(), dt_in, dt_next, times, true,
                    (cudaStream_t)stream);
}

int wm_batch_info(wm_batch* b, int* nblocks, int* ntiles, long long* launches_per_step) {
    if (!b) return fail(WM_E_INVALID, "null batch");
    const View& v = b->view;
    int inflow = 0;
    for (wm_case* c : v.members) inflow += c->has_inflow ? 1 : 0;
    const long long per_stage = IN_LAUNCHES * inflow + ((v.total_rhs || !v.hw.empty() || v.any_sponge) ? 1 : 0) + 1;
    if (nblocks) *nblocks = v.nblocks;
    if (ntiles) *ntiles = (int)v.tiles.size();
    if (launches_per_step) *launches_per_step = 3 * per_stage + 1;
    return WM_OK;
}

int wm_profile_enable(wm_case* c, int enable) {
    if (!c) return fail(WM_E_INVALID, "null case");
    c->prof.reset(enable != 0);
    return WM_OK;
}

int wm_profile_read(wm_case* c, int kind, double* ms_total, long long* launches) {
    if (!c || kind < -1 || kind >= WM_NKINDS) return fail(WM_E_INVALID, "bad profile query");
    double ms = 0.0;
    for (auto& r : c->prof.recs) {
        if (kind >= 0 && r.kind != kind) continue;
        CK(cudaEventSynchronize(r.b));
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, r.a, r.b));
        ms += t;
    }
    long long n = 0;
    for (int k = 0; k < WM_NKINDS; ++k)
        if (kind < 0 || k == kind) n += c->prof.nlaunch[k];
    if (ms_total) *ms_total = ms;
    if (launches) *launches = n;
    return WM_OK;
}

}  // extern "C"
