// Fused RHS + SSP-RK3 stage kernel.
//
// One CTA owns a TJ x TK tile of (j,k) columns of one block and marches along i over a
// chunk of planes [i0, i1).  Shared memory holds
//   pr[5]  primitive records of planes i-2..i+2 on the tile + 2-cell halo (rolling ring;
//          four slots, planes i-2..i+1, in the float form and the tiles that run several
//          CTAs per SM)
//   qs     the conservative values of the next plane to convert on the same footprint,
//          arriving by cp.async while plane i is being computed
//   gs     Green-Gauss gradients, mu_eff, k_eff (and the Ducros sensor) of plane i on the
//          tile + 1-cell halo
//   fj/fk  the j- and k-face fluxes of plane i
// and registers, per column, the previous i-face flux, the j/k flux differences of the
// previous plane and that plane's gradient record.  Per plane there are two phases
// separated by barriers:
//   1. gradient records of plane i; the warps without a record convert the staged plane
//      i+2 to primitives
//   2. own i-face flux -> RK epilogue of plane i-1; all j/k faces of plane i (flat loop);
//      the cp.async of plane i+3 is in flight meanwhile (KEP: the epilogue of plane i-1 runs
//      in the next phase 1 instead, on the warps without a gradient record)
// (float form, or several CTAs per SM: three phases, the conversion of plane i+1 first and
// on its own).
// Each face flux is evaluated once; each conservative value is read from HBM about once
// per stage (halo re-reads hit L2).  Stage 3 also emits per-(column, plane) partial sums of
// rho u V for the constant-mass-flux constraint.
//
// Reference: Solver._block_rhs (wmles/solver.py:76-95), green_gauss / viscous_flux /
// ducros (wmles/viscous.py), schemes (wmles/schemes.py), SGS (wmles/sgs.py), SSP-RK3
// (wmles/solver.py:110-121).
#include <cstdio>
#include <type_traits>
#include "physics.cuh"
#include "stage.cuh"

namespace wm {

// resident CTAs per SM the register budget is sized for: the FP64 form of the 256-thread
// tiles needs ~250 registers and 170+ KB of shared memory (one CTA); the float form fits
// two 256-thread CTAs (<= 128 registers, ~96 KB each), three 128-thread CTAs, or one
// 512-thread CTA
constexpr int stage_min_ctas(size_t rsize, int nt) {
    return rsize == 4 ? (nt <= 128 ? 3 : (nt <= 256 ? 2 : 1)) : (nt <= 128 ? 2 : 1);
}

// warps per CTA beyond the tile's columns: they take a share of every flat loop (primitive
// conversion, gradient records, j/k faces), so a plane's rounds of work are fuller and more
// warps hide the FP64 latency; the column-bound work (i-face flux, RK epilogue) stays with
// the first TJ x TK threads.  FP64 256-column tiles only, where one CTA per SM is resident.
// The launch bound of the larger CTA holds the kernel at 168 (352 threads) or 128 registers
// (448, 512 threads), with up to ~580 B of spills at 128, and it is still faster.  Measured
// stage time per step, 8 x 32 tile (channel 256x128x128 KEP / smooth ramp 384x96x64 / NACA
// C-grid 576x64x40, Hybrid): 3.17 / 3.37 /
// 3.72 ms at 256 threads (254 registers), 2.81 / 3.08 / 3.74 at 352, 2.65 / 2.81 / 3.20 at
// 448, 2.67 / 2.78 / 3.03 at 512; 16 x 16 tile: KEP 2.93 at 448 (3.03 at 352), Hybrid
// 3.12 / 2.61 at 352 (3.17 / 2.77 at 384, 3.52 / 2.85 at 512).  Since the FP64 form's two
// phases per plane (below), KEP runs 512 threads as well: 16 warps are charged the registers
// of 14 (groups of four), and the conversion gets five warps (channel stage per step 2.586
// against 2.598 ms at 448).  The float form's two-CTA
// tiles (issue-bound rather than latency-bound) gain nothing measurable and keep their
// columns' threads; its one-CTA 16 x 32 tile runs 640 threads at 96 registers (mixed stage
// time per step, channel / ramp / C-grid: 1.52 / 1.23 / 1.14 ms, against 1.65 / 1.36 / 1.23 at
// 512 threads and 1.58 / 1.31 / 1.21 for the best two-CTA tile).
constexpr int STAGE_MAX_WARPS = 32;          // two reduction sums per warp in the scratch
constexpr int stage_extra_warps(size_t rsize, int scheme, int tj, int tk) {
    if (rsize == 4) return tj * tk == 512 ? 4 : 0;
    if (tj * tk != 256) return 0;
    if (scheme == WM_SCHEME_KEP) return 8;
    return tj == 8 ? 8 : 3;
}

template <typename R, int SCHEME, int TJ, int TK>
struct StageLayout {
    static constexpr int NT = TJ * TK;                                         // tile columns
    static constexpr int NTH = NT + 32 * stage_extra_warps(sizeof(R), SCHEME, TJ, TK);   // threads
    static constexpr int PJ = TJ + 4, PK = TK + 4, PN = PJ * PK;   // primitives: 2-cell halo
    static constexpr int GJ = TJ + 2, GK = TK + 2, GN = GJ * GK;   // gradients: 1-cell halo
    static constexpr int NGS = (SCHEME == WM_SCHEME_HYBRID) ? 15 : 14;
    static constexpr int FJN = (TJ + 1) * TK, FKN = TJ * (TK + 1);
    // resident CTAs per SM the register budget is sized for: the FP64 form of the 256-thread
    // tiles needs ~250 registers and 170+ KB of shared memory (one CTA); the float form
    // fits two 256-thread CTAs (<= 128 registers, ~96 KB each) or three 128-thread CTAs
    static constexpr int MIN_CTAS = stage_min_ctas(sizeof(R), NTH);
    // FP64, one CTA per SM: a fifth primitive slot (the shared memory is there), so plane
    // i+2 is converted while the gradient records of plane i are computed, by the warps that
    // have no record to compute, and a plane takes two barriers instead of three.  FP64 stage
    // time per step, channel 256x128x128 / smooth ramp 384x96x64 / NACA C-grid 576x64x40:
    // 2.62 / 2.63 / 2.91 ms against 2.70 / 2.75 / 2.93 with three phases.  The float
    // form's one-CTA 16 x 32 tile has a record for nearly every thread (612 records, 640
    // threads) and gains nothing (ramp / C-grid 1.17 / 1.09 ms against 1.17 / 1.08): it keeps
    // three phases.
    static constexpr bool FUSE = MIN_CTAS == 1 && sizeof(R) == 8;
    static constexpr int NSLOT = FUSE ? 5 : 4;
    // KEP in the two-phase form: the RK epilogue deferred to the next gradient phase (below).
    // Channel 256x128x128 stage per step 2.546 ms against 2.583; the Hybrid kernels, whose gradient phase
    // is the longer one, lose with it (ramp +0.5 %, C-grid +6.4 %) and keep it in the face phase.
    static constexpr bool DEFER = FUSE && SCHEME == WM_SCHEME_KEP;
    static constexpr size_t qs_off = 0;                                        // double [5][PN]
    static constexpr size_t pr_off = qs_off + sizeof(double) * 5 * PN;         // R [NSLOT][PR_N][PN]
    static constexpr size_t gs_off = pr_off + sizeof(R) * NSLOT * PR_N * PN;   // R [NGS][GN]
    static constexpr size_t fj_off = gs_off + sizeof(R) * NGS * GN;            // R [5][FJN]
    static constexpr size_t fk_off = fj_off + sizeof(R) * 5 * FJN;             // R [5][FKN]
    // deferred epilogue: the flux divergence of the output plane per tile column
    static constexpr size_t fr_off = fk_off + sizeof(R) * 5 * FKN;            // R [5][NT]
    static constexpr size_t red_off = (fr_off + (DEFER ? sizeof(R) * 5 * NT : 0) + 15) / 16 * 16;
    static constexpr size_t bytes = red_off + sizeof(double) * 2 * STAGE_MAX_WARPS;
    static_assert(NTH / 32 <= STAGE_MAX_WARPS, "the reduction scratch holds two sums per warp");
    static_assert(!FUSE || GN <= NTH, "the fused phase computes one gradient record per thread");
    static_assert(bytes <= 227 * 1024, "shared memory of one CTA");
};

// gradient record: g[0..11] = d(u,v,w,T)/d(x,y,z), 12 = mu_eff, 13 = k_eff (all at half
// scale), 14 = theta
enum { GS_MU = 12, GS_K = 13, GS_TH = 14 };

// metric component arrays in the compute precision
template <typename R>
__device__ __forceinline__ const R* metbase(const BlockDev& B) {
    if constexpr (sizeof(R) == 4) return B.met32;
    else return B.met;
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];\n" ::"l"(p)); }
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p)); }

// viscous flux through one face (times area), wmles/viscous.py:28-51.  gL/gR index a
// gradient record (half scale: the face average of two records is their sum, the same
// value bit for bit as 0.5 (a + b), since scaling by two is exact); pl/pr point at primitive
// records with component stride s; (e0, e1, e2) is the unit vector from the L to the R cell
// centre and idist the inverse distance.
template <typename R, class GL, class GR>
__device__ __forceinline__ void viscous_flux(const R* pl, const R* pr, int s, GL gL, GR gR, R Sx, R Sy, R Sz,
                                             R e0, R e1, R e2, R idist, R F[5]) {
    R gf[12];
    const int pv[4] = {PR_U, PR_V, PR_W, PR_T};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const R b0 = gL(3 * a) + gR(3 * a);
        const R b1 = gL(3 * a + 1) + gR(3 * a + 1);
        const R b2 = gL(3 * a + 2) + gR(3 * a + 2);
        const R corr = (pr[pv[a] * s] - pl[pv[a] * s]) * idist - (b0 * e0 + b1 * e1 + b2 * e2);
        gf[3 * a] = b0 + corr * e0;
        gf[3 * a + 1] = b1 + corr * e1;
        gf[3 * a + 2] = b2 + corr * e2;
    }
    const R div = gf[0] + gf[4] + gf[8];
    const R muf = gL(GS_MU) + gR(GS_MU);
    const R kf = gL(GS_K) + gR(GS_K);
    const R d23 = R(2.0 / 3.0) * div;
    const R t00 = muf * (gf[0] + gf[0] - d23), t11 = muf * (gf[4] + gf[4] - d23), t22 = muf * (gf[8] + gf[8] - d23);
    const R t01 = muf * (gf[1] + gf[3]), t02 = muf * (gf[2] + gf[6]), t12 = muf * (gf[5] + gf[7]);
    const R ts0 = t00 * Sx + t01 * Sy + t02 * Sz;
    const R ts1 = t01 * Sx + t11 * Sy + t12 * Sz;
    const R ts2 = t02 * Sx + t12 * Sy + t22 * Sz;
    const R dTdn = gf[9] * Sx + gf[10] * Sy + gf[11] * Sz;
    const R uf = R(0.5) * (pl[PR_U * s] + pr[PR_U * s]);
    const R vf = R(0.5) * (pl[PR_V * s] + pr[PR_V * s]);
    const R wf = R(0.5) * (pl[PR_W * s] + pr[PR_W * s]);
    F[1] -= ts0;
    F[2] -= ts1;
    F[3] -= ts2;
    F[4] -= (uf * ts0 + vf * ts1 + wf * ts2) + kf * dTdn;
}

// total face flux (inviscid scheme + viscous), S = face area vector, e / idist = unit
// centre-to-centre vector and its inverse length
template <typename R, int SCHEME, class GL, class GR>
__device__ __forceinline__ void face_flux(const StageOpts& o, const Phys<R>& P, const R* L2, const R* L,
                                          const R* Rr, const R* R2, int s, GL gL, GR gR, R Sx, R Sy,
                                          R Sz, R e0, R e1, R e2, R idist, R F[5]) {
    if constexpr (SCHEME == WM_SCHEME_KEP) {
        kep_flux(o.kep_order, L2, L, Rr, R2, s, Sx, Sy, Sz, F);
    } else if constexpr (SCHEME == WM_SCHEME_MUSCL) {
        muscl_hllc_flux(o.limiter, L2, L, Rr, R2, s, Sx, Sy, Sz, P, F);
    } else {
        // Ducros-switched blend, wmles/schemes.py:163-166
        const R th = fmax(gL(GS_TH), gR(GS_TH));
        const R sw = fmin(fmax((th - P.th0) * P.inv_dth, R(0)), R(1));
        R Fc[5] = {R(0), R(0), R(0), R(0), R(0)}, Fu[5] = {R(0), R(0), R(0), R(0), R(0)};
        if (sw < R(1)) kep_flux(o.kep_order, L2, L, Rr, R2, s, Sx, Sy, Sz, Fc);
        if (sw > R(0)) muscl_hllc_flux(o.limiter, L2, L, Rr, R2, s, Sx, Sy, Sz, P, Fu);
#pragma unroll
        for (int v = 0; v < 5; ++v) F[v] = (sw == R(0)) ? Fc[v] : (sw == R(1)) ? Fu[v] : (R(1) - sw) * Fc[v] + sw * Fu[v];
    }
    viscous_flux<R>(L, Rr, s, gL, gR, Sx, Sy, Sz, e0, e1, e2, idist, F);
}

// one segment of a CTA's work: tile t (a (j,k) column of one block over planes [t.i0, t.i1))
template <typename R, int SCHEME, int TJ, int TK>
__device__ __forceinline__ void stage_segment(const StageArgs& A, const StageOpts& o, const Tile t,
                                              unsigned char* smem_raw) {
    using LY = StageLayout<R, SCHEME, TJ, TK>;
    constexpr int NT = LY::NT, NTH = LY::NTH, PK = LY::PK, PN = LY::PN, GK = LY::GK, GN = LY::GN, NGS = LY::NGS;
    double* qs = reinterpret_cast<double*>(smem_raw + LY::qs_off);
    R* pr = reinterpret_cast<R*>(smem_raw + LY::pr_off);
    R* gs = reinterpret_cast<R*>(smem_raw + LY::gs_off);
    R* fj = reinterpret_cast<R*>(smem_raw + LY::fj_off);
    R* fk = reinterpret_cast<R*>(smem_raw + LY::fk_off);
    R* fr = reinterpret_cast<R*>(smem_raw + LY::fr_off);
    double* red = reinterpret_cast<double*>(smem_raw + LY::red_off);

    const BlockDev B = A.blocks[t.blk];
    const CaseDev& C = A.cases[B.case_id];
    const Phys<R> P(C);
    const StatePtrs SP = A.p[t.blk];
    const int ng = B.ng, Nj = B.N[1], Nk = B.N[2];
    const long long plane = B.plane, ncell = B.ncell;
    // cell and component offsets fit 32 bits (checked at case creation): one base pointer
    // per cell, 32-bit offsets per component
    const int planei = (int)B.plane, nc = (int)B.ncell;
    const R* MB = metbase<R>(B);
    const int tid = threadIdx.x, tj = tid / TK, tk = tid % TK;
    const int jhi = ng + B.n[1], khi = ng + B.n[2], ihi = ng + B.n[0];
    const int j = t.j0 + tj, k = t.k0 + tk;
    const bool column = tid < NT;                  // this thread owns a tile column
    // j/k-face loop index: the extra warps (no i-face flux of their own) come first, so the
    // face work of a plane is spread more evenly over the threads
    const int rtid = column ? tid + (NTH - NT) : tid - NT;
    const bool active = column && (j < jhi) && (k < khi);
    const int sgs_model = o.sgs;

    // ---- conservative values of plane ip on the tile + 2-cell halo -> staging buffer (async)
    auto stage_plane = [&](int ip) {
        for (int c = tid; c < PN; c += NTH) {
            const int jj = c / PK, kk = c - jj * PK;
            const int gj = min(max(t.j0 - 2 + jj, 0), Nj - 1);
            const int gk = min(max(t.k0 - 2 + kk, 0), Nk - 1);
            const int idx = ip * planei + gj * Nk + gk;
#pragma unroll
            for (int v = 0; v < 5; ++v) cp_async8(qs + v * PN + c, SP.q_in + v * nc + idx);
        }
    };
    // ring slot of plane ip's primitive records
    auto slot = [](int ip) { return LY::FUSE ? ip % LY::NSLOT : ip & 3; };
    // ---- staged value c -> primitive record c of plane ip
    auto convert_cell = [&](int ip, int c) {
        R* dst = pr + slot(ip) * PR_N * PN;
        double q[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) q[v] = qs[v * PN + c];
        R rec[PR_N];
        cons_to_rec(q, P, rec);
#pragma unroll
        for (int v = 0; v < PR_N; ++v) dst[v * PN + c] = rec[v];
    };
    auto convert_plane = [&](int ip) {
        for (int c = tid; c < PN; c += NTH) convert_cell(ip, c);
    };

    // ---- gradient record c of plane ip (ring slots of ip-1, ip, ip+1) on the tile + 1-cell halo
    auto grad_cell = [&](int ip, int c) {
        const R* Pm = pr + slot(ip - 1) * PR_N * PN;
        const R* P0 = pr + slot(ip) * PR_N * PN;
        const R* Pp = pr + slot(ip + 1) * PR_N * PN;
        {
            const int jj = c / GK, kk = c - jj * GK;
            const int pc = (jj + 1) * PK + (kk + 1);
            const int gj = min(t.j0 - 1 + jj, Nj - 2), gk = min(t.k0 - 1 + kk, Nk - 2);
            const int pv[4] = {PR_U, PR_V, PR_W, PR_T};
            // metrics first: their loads overlap
            const R* m = MB + (ip * planei + gj * Nk + gk);
            const R* mi = m + planei;
            const R* mj = m + Nk;
            const R* mk = m + 1;
            const R Six = __ldg(m + WM_MET_SIX * nc), Siy = __ldg(m + WM_MET_SIY * nc), Siz = __ldg(m + WM_MET_SIZ * nc);
            const R Hix = __ldg(mi + WM_MET_SIX * nc), Hiy = __ldg(mi + WM_MET_SIY * nc), Hiz = __ldg(mi + WM_MET_SIZ * nc);
            const R Sjx = __ldg(m + WM_MET_SJX * nc), Sjy = __ldg(m + WM_MET_SJY * nc), Sjz = __ldg(m + WM_MET_SJZ * nc);
            const R Hjx = __ldg(mj + WM_MET_SJX * nc), Hjy = __ldg(mj + WM_MET_SJY * nc), Hjz = __ldg(mj + WM_MET_SJZ * nc);
            const R Skx = __ldg(m + WM_MET_SKX * nc), Sky = __ldg(m + WM_MET_SKY * nc), Skz = __ldg(m + WM_MET_SKZ * nc);
            const R Hkx = __ldg(mk + WM_MET_SKX * nc), Hky = __ldg(mk + WM_MET_SKY * nc), Hkz = __ldg(mk + WM_MET_SKZ * nc);
            // a quarter of 1/V: the face values below are sums of two cells, twice the face
            // averages (scaling by two is exact, so the products and sums are the averages'
            // bit for bit, doubled), and the record holds half the gradient (faces average two
            // records by adding them); the SGS models are homogeneous of degree one in the
            // gradient and the Ducros sensor of degree zero, so they take the half gradient
            const R qivol = R(0.25) * __ldg(m + WM_MET_IVOL * nc);
            const R delta = sgs_model != WM_SGS_NONE ? __ldg(m + WM_MET_DELTA * nc) : R(0);
            R acc[12];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const R c0 = P0[pv[a] * PN + pc];
                const R li = Pm[pv[a] * PN + pc] + c0, hi = c0 + Pp[pv[a] * PN + pc];
                const R lj = P0[pv[a] * PN + pc - PK] + c0, hj = c0 + P0[pv[a] * PN + pc + PK];
                const R lk = P0[pv[a] * PN + pc - 1] + c0, hk = c0 + P0[pv[a] * PN + pc + 1];
                acc[3 * a] = ((hi * Hix - li * Six) + (hj * Hjx - lj * Sjx)) + (hk * Hkx - lk * Skx);
                acc[3 * a + 1] = ((hi * Hiy - li * Siy) + (hj * Hjy - lj * Sjy)) + (hk * Hky - lk * Sky);
                acc[3 * a + 2] = ((hi * Hiz - li * Siz) + (hj * Hjz - lj * Sjz)) + (hk * Hkz - lk * Skz);
            }
#pragma unroll
            for (int q = 0; q < 12; ++q) acc[q] *= qivol;
            const R T = P0[PR_T * PN + pc];
            const R muh = R(0.5) * sutherland(T, P);              // half the molecular viscosity
            R muth = R(0);                                        // half the eddy viscosity
            if (sgs_model != WM_SGS_NONE) {
                const R rho = P0[PR_RHO * PN + pc];
                muth = rho * sgs_nut(sgs_model, acc, delta, P.sgs_c);
            }
#pragma unroll
            for (int q = 0; q < 12; ++q) gs[q * GN + c] = acc[q];
            gs[GS_MU * GN + c] = muh + muth;
            gs[GS_K * GN + c] = P.cp * (muh * P.inv_Pr + muth * P.inv_Prt);
            if constexpr (NGS > 14) gs[GS_TH * GN + c] = ducros(acc);
        }
    };
    auto grad_plane = [&](int ip) {
        for (int c = tid; c < GN; c += NTH) grad_cell(ip, c);
    };
    // ---- gradient records of plane ip and (conv) primitives of plane ip+2 from the staging
    // buffer.  The warps that hold a record take one each; the warps left over convert (at
    // most five cells each, about the time of one record), and the cells beyond their share
    // go to the record warps after their record.  (The 8 x 32 tile at 512 threads: 160
    // converting threads, three rounds.  At 448 threads, 96 converting threads: five rounds
    // took every cell; three or four rounds with the rest on the record warps were 1.1-1.4 %
    // slower on the channel, the same on the ramp and the C-grid.)
    auto grad_convert = [&](int ip, bool conv) {
        constexpr int GW = (GN + 31) / 32 * 32;          // threads of the record warps
        constexpr int SP = NTH - GW;                     // threads of the converting warps
        constexpr int CR = SP > 0 ? (PN + SP - 1) / SP < 5 ? (PN + SP - 1) / SP : 5 : 0;
        constexpr int CS = SP * CR;                      // cells the converting warps take
        if (tid < GW) {
            if (tid < GN) grad_cell(ip, tid);
            if (conv)
                for (int c = CS + tid; c < PN; c += GW) convert_cell(ip + 2, c);
        } else if (conv) {
            for (int c = tid - GW; c < CS && c < PN; c += SP) convert_cell(ip + 2, c);
        }
    };

    // wall-model flux override of face (axis, side) at tangential position (a, b)
    auto wall_flux = [&](int face, int a, int b, R F[5]) -> bool {
        const int w = B.wall[face];
        if (w < 0) return false;
        const WallDev& W = A.walls[w];
        const long long f = (long long)(a - ng) * W.nt2 + (b - ng);
        const long long nf = (long long)W.nt1 * W.nt2;
#pragma unroll
        for (int v = 0; v < 5; ++v) F[v] = R(W.F[v * nf + f]);
        return true;
    };

    // ---- i-face flux between planes ip-1 and ip for this thread's column
    R gsp[NGS];   // gradient record of plane ip-1 at this column
#pragma unroll
    for (int v = 0; v < NGS; ++v) gsp[v] = R(0);
    auto iface_flux = [&](int ip, R F[5]) {
        if (ip == ng && wall_flux(0, j, k, F)) return;
        if (ip == ihi && wall_flux(1, j, k, F)) return;
        const int pc = (tj + 2) * PK + (tk + 2);
        const int gc = (tj + 1) * GK + (tk + 1);
        const R* L2 = pr + slot(ip - 2) * PR_N * PN + pc;
        const R* L = pr + slot(ip - 1) * PR_N * PN + pc;
        const R* Rr = pr + slot(ip) * PR_N * PN + pc;
        const R* R2 = pr + slot(ip + 1) * PR_N * PN + pc;
        const R* m = MB + (ip * planei + j * Nk + k);
        const R Sx = __ldg(m + WM_MET_SIX * nc), Sy = __ldg(m + WM_MET_SIY * nc), Sz = __ldg(m + WM_MET_SIZ * nc);
        const R e0 = __ldg(m + WM_MET_EIX * nc), e1 = __ldg(m + WM_MET_EIY * nc), e2 = __ldg(m + WM_MET_EIZ * nc);
        const R id = __ldg(m + WM_MET_IDI * nc);
        face_flux<R, SCHEME>(o, P, L2, L, Rr, R2, PN, [&](int v) { return gsp[v]; },
                             [&](int v) { return gs[v * GN + gc]; }, Sx, Sy, Sz, e0, e1, e2, id, F);
    };

    // ---- one j- (f < FJN) or k-face flux of plane ip into shared memory
    auto jk_face = [&](int ip, int f) {
        const R* P0 = pr + slot(ip) * PR_N * PN;
        R F[5] = {R(0), R(0), R(0), R(0), R(0)};
        if (f < LY::FJN) {
            const int row = f / TK, kk = f - row * TK;
            const int gj = t.j0 + row, gk = t.k0 + kk;
            if (gj <= jhi && gk < khi) {
                bool done = false;
                if (gj == ng) done = wall_flux(2, ip, gk, F);
                else if (gj == jhi) done = wall_flux(3, ip, gk, F);
                if (!done) {
                    const int pc = (row + 2) * PK + (kk + 2);     // R cell in the primitive tile
                    const int gc = (row + 1) * GK + (kk + 1);     // R cell in the gradient tile
                    const R* m = MB + (ip * planei + gj * Nk + gk);
                    const R Sx = __ldg(m + WM_MET_SJX * nc), Sy = __ldg(m + WM_MET_SJY * nc), Sz = __ldg(m + WM_MET_SJZ * nc);
                    const R e0 = __ldg(m + WM_MET_EJX * nc), e1 = __ldg(m + WM_MET_EJY * nc);
                    const R e2 = __ldg(m + WM_MET_EJZ * nc), id = __ldg(m + WM_MET_IDJ * nc);
                    face_flux<R, SCHEME>(o, P, P0 + pc - 2 * PK, P0 + pc - PK, P0 + pc, P0 + pc + PK, PN,
                                         [&](int v) { return gs[v * GN + gc - GK]; },
                                         [&](int v) { return gs[v * GN + gc]; }, Sx, Sy, Sz, e0, e1, e2, id, F);
                }
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) fj[v * LY::FJN + f] = F[v];
        } else {
            f -= LY::FJN;
            const int row = f / (TK + 1), col = f - row * (TK + 1);
            const int gj = t.j0 + row, gk = t.k0 + col;
            if (gj < jhi && gk <= khi) {
                bool done = false;
                if (gk == ng) done = wall_flux(4, ip, gj, F);
                else if (gk == khi) done = wall_flux(5, ip, gj, F);
                if (!done) {
                    const int pc = (row + 2) * PK + (col + 2);
                    const int gc = (row + 1) * GK + (col + 1);
                    const R* m = MB + (ip * planei + gj * Nk + gk);
                    const R Sx = __ldg(m + WM_MET_SKX * nc), Sy = __ldg(m + WM_MET_SKY * nc), Sz = __ldg(m + WM_MET_SKZ * nc);
                    const R e0 = __ldg(m + WM_MET_EKX * nc), e1 = __ldg(m + WM_MET_EKY * nc);
                    const R e2 = __ldg(m + WM_MET_EKZ * nc), id = __ldg(m + WM_MET_IDK * nc);
                    face_flux<R, SCHEME>(o, P, P0 + pc - 2, P0 + pc - 1, P0 + pc, P0 + pc + 1, PN,
                                         [&](int v) { return gs[v * GN + gc - 1]; },
                                         [&](int v) { return gs[v * GN + gc]; }, Sx, Sy, Sz, e0, e1, e2, id, F);
                }
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) fk[v * LY::FKN + f] = F[v];
        }
    };

    // ---- cache-line prefetch of what the next plane reads from global memory: the metrics
    // of plane ip+1 on the gradient footprint (+1 row/column for upper faces), the i-face
    // areas of plane ip+2, and (stages 2, 3) the step-start state of plane ip on the tile
    auto prefetch_next = [&](int ip) {
        using MT = typename std::conditional<sizeof(R) == 4, float, double>::type;
        const MT* mbase = sizeof(R) == 4 ? reinterpret_cast<const MT*>(B.met32) : reinterpret_cast<const MT*>(B.met);
        constexpr int EL = sizeof(MT);
        constexpr int ROWS = TJ + 3, LINES = ((TK + 3) * EL + 127) / 128 + 1;
        const int r0 = t.j0 - 1, c0 = t.k0 - 1;
        // components read by the stage kernel: S (0..8), delta, 1/V, e/idist (13..26) of plane
        // ip+1 (23), then S_i (0..2) of plane ip+2 (3)
        constexpr int NPF = 26;
        for (int it = tid; it < NPF * ROWS * LINES; it += NTH) {
            const int comp = it / (ROWS * LINES), rem = it - comp * (ROWS * LINES);
            const int row = rem / LINES, line = rem - row * LINES;
            const int pl = comp < 23 ? ip + 1 : ip + 2;
            const int cc = comp < 9 ? comp : (comp < 23 ? comp + 4 : comp - 23);
            const int gj = min(r0 + row, Nj - 1);
            if (pl >= B.N[0]) continue;
            const MT* rowp = mbase + cc * ncell + (long long)pl * plane + (long long)gj * Nk;
            const uintptr_t a = (reinterpret_cast<uintptr_t>(rowp + c0) & ~uintptr_t(127)) + 128u * line;
            if (a <= reinterpret_cast<uintptr_t>(rowp + min(c0 + TK + 2, Nk - 1))) prefetch_l1(reinterpret_cast<const void*>(a));
        }
        if (A.stage >= 2 && ip < ihi) {
            constexpr int QL = (TK * 8 + 127) / 128 + 1;
            for (int it = tid; it < 5 * TJ * QL; it += NTH) {
                const int v = it / (TJ * QL), rem = it - v * (TJ * QL);
                const int row = rem / QL, line = rem - row * QL;
                const int gj = min(t.j0 + row, Nj - 1);
                const double* rowp = SP.q0 + v * ncell + (long long)ip * plane + (long long)gj * Nk;
                const uintptr_t a = (reinterpret_cast<uintptr_t>(rowp + t.k0) & ~uintptr_t(127)) + 128u * line;
                if (a <= reinterpret_cast<uintptr_t>(rowp + min(t.k0 + TK - 1, Nk - 1))) prefetch_l2(reinterpret_cast<const void*>(a));
            }
        }
    };

    auto save_gs = [&]() {
        if (!column) return;
        const int gc = (tj + 1) * GK + (tk + 1);
#pragma unroll
        for (int v = 0; v < NGS; ++v) gsp[v] = gs[v * GN + gc];
    };

    R dFj[5], dFk[5], Flo[5];
    auto jk_diff = [&]() {
        if (!column) return;
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            dFj[v] = fj[v * LY::FJN + (tj + 1) * TK + tk] - fj[v * LY::FJN + tj * TK + tk];
            dFk[v] = fk[v * LY::FKN + tj * (TK + 1) + tk + 1] - fk[v * LY::FKN + tj * (TK + 1) + tk];
        }
    };

    const int i0 = t.i0, i1 = t.i1;
    const double dt = A.stage ? *A.dt[B.case_id] : 0.0;
    // constant mass flux (stage 3): one partial of rho u_dir V per (tile column, plane) -
    // the warps' sums of the plane added in warp order in shared memory - so the case's sum
    // does not depend on how the columns are cut into chunks along i
    const bool cmf_on = A.stage == 3 && A.cmf_part != nullptr && C.cmf_dir >= 0;
    double cmf_acc = 0.0;
    double* cmf_col = nullptr;
    if (cmf_on) {
        const int ncolk = (B.n[2] + TK - 1) / TK;
        const int col = ((t.j0 - ng) / TJ) * ncolk + (t.k0 - ng) / TK;
        cmf_col = A.cmf_part + A.cmf_slot_start[t.blk] + (long long)col * B.n[0];
    }

    // ---- RK epilogue of interior cell (io, jj, kk) from its flux divergence dv (times -1, not
    // yet divided by V): r = -(div F)/V (+ source), stage update
    auto output = [&](int io, int jj, int kk, const R dv[5]) {
        const int idx = io * planei + jj * Nk + kk;
        const R ivol = __ldg(MB + WM_MET_IVOL * nc + idx);
        R r[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) r[v] = dv[v] * ivol;
        double rq[5], qi[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) qi[v] = __ldg(SP.q_in + v * nc + idx);
        if (C.sponge) {
            // -sigma(x) (q - spanwise mean), wmles/smooth_ramp.py:212-221
            const double xl = __ldg(B.met + WM_MET_XCX * nc + idx) * C.sp_invL;
            const double eta = fmin(fmax((xl - C.sp_xs) * C.sp_inv_dx, 0.0), 1.0);
            const double sig = C.sp_sigma0 * (eta * eta * eta * (10.0 + eta * (-15.0 + 6.0 * eta)));
            const long long mi = (long long)io * Nj + jj;
            const long long mn = (long long)B.N[0] * Nj;
#pragma unroll
            for (int v = 0; v < 5; ++v) rq[v] = double(r[v]) - sig * (qi[v] - SP.spmean[v * mn + mi]);
        } else {
#pragma unroll
            for (int v = 0; v < 5; ++v) rq[v] = double(r[v]);
        }
        if (A.stage == 0) {
#pragma unroll
            for (int v = 0; v < 5; ++v) SP.q_out[v * nc + idx] = rq[v];
        } else if (A.stage == 1) {
#pragma unroll
            for (int v = 0; v < 5; ++v) SP.q_out[v * nc + idx] = qi[v] + dt * rq[v];
        } else if (A.stage == 2) {
#pragma unroll
            for (int v = 0; v < 5; ++v)
                SP.q_out[v * nc + idx] = 0.75 * __ldg(SP.q0 + v * nc + idx) + 0.25 * (qi[v] + dt * rq[v]);
        } else {
            double qn[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                qn[v] = (1.0 / 3.0) * __ldg(SP.q0 + v * nc + idx) + (2.0 / 3.0) * (qi[v] + dt * rq[v]);
                SP.q_out[v * nc + idx] = qn[v];
            }
            if (C.cmf_dir >= 0) cmf_acc += qn[1 + C.cmf_dir] * __ldg(B.met + WM_MET_VOL * nc + idx);
        }
    };

    // ---- L1 prefetch of what the RK epilogue of plane io reads at this thread's cell, issued
    // before the i-face flux.  KEP scheme only: channel FP64 stage per step 2.59 ms against
    // 2.62; the Hybrid kernels (ramp, C-grid), which spill more, lose 1-2 % to the extra L1
    // lines.  Loading these values into registers ahead of the flux instead spills more and is
    // slower in every case.
    auto prefetch_epilogue = [&](int io, int jj, int kk) {
        const int idx = io * planei + jj * Nk + kk;
        prefetch_l1(MB + WM_MET_IVOL * nc + idx);
#pragma unroll
        for (int v = 0; v < 5; ++v) prefetch_l1(SP.q_in + v * nc + idx);
        if (A.stage >= 2)
#pragma unroll
            for (int v = 0; v < 5; ++v) prefetch_l1(SP.q0 + v * nc + idx);
        if (cmf_on) prefetch_l1(B.met + WM_MET_VOL * nc + idx);
    };

    // ---- deferred epilogue (KEP, FP64 two-phase form): the RK epilogue of plane io runs in the
    // gradient phase of the plane after next (its flux divergence waits in fr), on the warps
    // that hold no gradient record (on every thread when there are none), so that the face
    // phase is no longer set by the column threads' i-face flux + epilogue + j/k face; stage
    // 3's rho u_dir V of the plane is summed per warp into red
    constexpr int EGW = (GN + 31) / 32 * 32, ESP = NTH - EGW;
    auto epi_cells = [&](auto&& f) {
        if constexpr (ESP >= 32) {
            if (tid >= EGW)
                for (int c = tid - EGW; c < NT; c += ESP) f(c);
        } else {
            for (int c = tid; c < NT; c += NTH) f(c);
        }
    };
    auto epilogue_plane = [&](int io) {
        epi_cells([&](int c) {
            const int jj = t.j0 + c / TK, kk = t.k0 + c % TK;
            if (jj < jhi && kk < khi) {
                R dv[5];
#pragma unroll
                for (int v = 0; v < 5; ++v) dv[v] = fr[v * NT + c];
                output(io, jj, kk, dv);
            }
        });
        if (cmf_on) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) cmf_acc += __shfl_down_sync(0xffffffffu, cmf_acc, off);
            if ((tid & 31) == 0) red[tid >> 5] = cmf_acc;
            cmf_acc = 0.0;
        }
    };
    auto cmf_store = [&](int io) {      // after the barrier that follows epilogue_plane(io)
        if (cmf_on && tid == 0) {
            double sp = 0.0;
            for (int w = 0; w < NTH / 32; ++w) sp += red[w];
            cmf_col[io - ng] = sp;
        }
    };

    // ---- prologue: planes i0-2 .. i0+1 (and i0+2 when fused), gradients of i0-1 and i0,
    // faces of plane i0
    constexpr int PRE = LY::FUSE ? 2 : 1;          // last plane converted ahead of the march
#pragma unroll 1
    for (int ip = i0 - 2; ip <= i0 + PRE; ++ip) {
        stage_plane(ip);
        cp_async_wait_all();
        __syncthreads();
        convert_plane(ip);
        __syncthreads();
    }
    if (i0 + PRE + 1 <= i1 + 1) stage_plane(i0 + PRE + 1);   // in flight during the prologue's compute
    grad_plane(i0 - 1);
    __syncthreads();
    save_gs();
    __syncthreads();
    grad_plane(i0);
    __syncthreads();
    if (active) iface_flux(i0, Flo);
    if constexpr (LY::FUSE) save_gs();   // before the barrier: no barrier precedes the next records
    for (int f = rtid; f < LY::FJN + LY::FKN; f += NTH) jk_face(i0, f);
    cp_async_wait_all();
    __syncthreads();
    jk_diff();
    if constexpr (!LY::FUSE) save_gs();

    // ---- march: iteration ip outputs plane ip-1
#pragma unroll 1
    for (int ip = i0 + 1; ip <= i1; ++ip) {
        if constexpr (LY::FUSE) {
            grad_convert(ip, ip < i1);   // records of plane ip; staged plane ip+2 -> primitives
            if constexpr (LY::DEFER)
                if (ip - 2 >= i0) epilogue_plane(ip - 2);
            __syncthreads();
            if constexpr (LY::DEFER)
                if (ip - 2 >= i0) cmf_store(ip - 2);
            if (ip + 3 <= i1 + 1) stage_plane(ip + 3);
        } else {
            convert_plane(ip + 1);       // staged plane ip+1 -> primitives
            __syncthreads();
            grad_plane(ip);
            __syncthreads();
            if (ip + 2 <= i1 + 1) stage_plane(ip + 2);
        }
        if constexpr (SCHEME == WM_SCHEME_KEP) {
            if constexpr (LY::DEFER) {
                epi_cells([&](int c) {
                    const int jj = t.j0 + c / TK, kk = t.k0 + c % TK;
                    if (jj < jhi && kk < khi) prefetch_epilogue(ip - 1, jj, kk);
                });
            } else if (active) {
                prefetch_epilogue(ip - 1, j, k);
            }
        }
        if (ip < i1) prefetch_next(ip);
        if (active) {
            R Fhi[5], dv[5];
            iface_flux(ip, Fhi);
#pragma unroll
            for (int v = 0; v < 5; ++v) dv[v] = (-(Fhi[v] - Flo[v]) - dFj[v]) - dFk[v];
            if constexpr (LY::DEFER) {
#pragma unroll
                for (int v = 0; v < 5; ++v) fr[v * NT + tid] = dv[v];
            } else {
                output(ip - 1, j, k, dv);
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) Flo[v] = Fhi[v];
        }
        if constexpr (LY::FUSE) save_gs();
        if (!LY::DEFER && cmf_on) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) cmf_acc += __shfl_down_sync(0xffffffffu, cmf_acc, off);
            // warp sums of this plane; two buffers by plane parity (read after the barrier below)
            if ((tid & 31) == 0) red[(ip & 1) * (NTH / 32) + (tid >> 5)] = cmf_acc;
            cmf_acc = 0.0;
        }
        if (ip < i1)
            for (int f = rtid; f < LY::FJN + LY::FKN; f += NTH) jk_face(ip, f);
        cp_async_wait_all();
        __syncthreads();
        if (!LY::DEFER && cmf_on && tid == 0) {
            double sp = 0.0;
            for (int w = 0; w < NTH / 32; ++w) sp += red[(ip & 1) * (NTH / 32) + w];
            cmf_col[ip - 1 - ng] = sp;
        }
        if (ip < i1) {
            jk_diff();
            if constexpr (!LY::FUSE) save_gs();
        }
    }
    if constexpr (LY::DEFER) {
        epilogue_plane(i1 - 1);          // the segment's last plane
        if (cmf_on) {
            __syncthreads();
            cmf_store(i1 - 1);
        }
    }
}

template <typename R, int SCHEME, int TJ, int TK>
__global__ void __launch_bounds__(StageLayout<R, SCHEME, TJ, TK>::NTH, StageLayout<R, SCHEME, TJ, TK>::MIN_CTAS)
    stage_kernel(const __grid_constant__ StageArgs A, const StageOpts o) {
    using LY = StageLayout<R, SCHEME, TJ, TK>;
    constexpr int NTH = LY::NTH;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* red = reinterpret_cast<double*>(smem_raw + LY::red_off);
    const int tid = threadIdx.x;
    // this CTA's segments: one tile, or a balanced range of tiles (consecutive column pieces)
    const int first = A.cta_first ? A.cta_first[blockIdx.x] : blockIdx.x;
    const int last = A.cta_first ? A.cta_first[blockIdx.x + 1] : blockIdx.x + 1;
#pragma unroll 1
    for (int ti = first; ti < last; ++ti) {
        stage_segment<R, SCHEME, TJ, TK>(A, o, A.tiles[ti], smem_raw);
        __syncthreads();                 // shared memory is reused by the next segment
    }

    if (A.stage == 3 && A.cmf_part != nullptr) {
        // every CTA of the launch signals; the last one reduces each case's partials
        __shared__ bool last_cta;
        if (tid == 0) __threadfence();
        __syncthreads();
        if (tid == 0) last_cta = atomicAdd(A.cmf_counter, 1u) == unsigned(gridDim.x - 1);
        __syncthreads();
        if (last_cta) {
            // per case: the sum over that case's partials in slot order (the same alone or in
            // a batch, for any chunk length, run to run) and the shift
            // delta = target - sum(rho u V) / sum(V), wmles/solver.py:24-29
            __threadfence();
            const volatile double* part = A.cmf_part;
            for (int c = 0; c < A.ncases; ++c) {
                const CaseDev& Cc = A.cases[c];
                if (Cc.cmf_dir < 0) continue;
                const int s0 = A.case_slot_start[c], s1 = A.case_slot_start[c + 1];
                double s = 0.0;
                for (int i = s0 + tid; i < s1; i += NTH) s += part[i];
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
                __syncthreads();
                if ((tid & 31) == 0) red[tid >> 5] = s;
                __syncthreads();
                if (tid == 0) {
                    double tot = 0.0;
                    for (int w = 0; w < NTH / 32; ++w) tot += red[w];
                    A.cmf_delta[c] = Cc.cmf_target - tot / Cc.cmf_volume;
                }
            }
            if (tid == 0) *A.cmf_counter = 0u;
        }
    }
}

template <typename R, int SCHEME, int TJ, int TK>
static cudaError_t configure_one() {
    using LY = StageLayout<R, SCHEME, TJ, TK>;
    static std::atomic<unsigned long long> done{0};     // per instantiation, one bit per device
    return once_per_device(done, [] {
        return cudaFuncSetAttribute(stage_kernel<R, SCHEME, TJ, TK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)LY::bytes);
    });
}

template <typename R, int SCHEME, int TJ, int TK>
static cudaError_t launch_one(const StageArgs& A, const StageOpts& o, cudaStream_t s) {
    using LY = StageLayout<R, SCHEME, TJ, TK>;
    cudaError_t e = configure_one<R, SCHEME, TJ, TK>();
    if (e != cudaSuccess) return e;
    stage_kernel<R, SCHEME, TJ, TK><<<A.nctas, LY::NTH, LY::bytes, s>>>(A, o);
    return cudaGetLastError();
}

template <typename R, int SCHEME, int TJ, int TK>
static int occupancy_one() {
    using LY = StageLayout<R, SCHEME, TJ, TK>;
    if (configure_one<R, SCHEME, TJ, TK>() != cudaSuccess) return 1;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage_kernel<R, SCHEME, TJ, TK>, LY::NTH, LY::bytes) !=
        cudaSuccess)
        return 1;
    return n;
}

// tile shapes: 0 = 8x32, 1 = 16x16, 2 = 4x32, 3 = 16x32 (float only)
template <typename R, int SCHEME>
static cudaError_t launch_tile(const StageArgs& A, const StageOpts& o, cudaStream_t s) {
    switch (o.tile) {
        case 1: return launch_one<R, SCHEME, 16, 16>(A, o, s);
        case 2: return launch_one<R, SCHEME, 4, 32>(A, o, s);
        case 3:
            if constexpr (sizeof(R) == 4) return launch_one<R, SCHEME, 16, 32>(A, o, s);
            else return cudaErrorInvalidValue;     // the FP64 16x32 tile exceeds shared memory
        default: return launch_one<R, SCHEME, 8, 32>(A, o, s);
    }
}

template <typename R, int SCHEME>
static int occupancy_tile(int tile) {
    switch (tile) {
        case 1: return occupancy_one<R, SCHEME, 16, 16>();
        case 2: return occupancy_one<R, SCHEME, 4, 32>();
        case 3:
            if constexpr (sizeof(R) == 4) return occupancy_one<R, SCHEME, 16, 32>();
            else return 0;
        default: return occupancy_one<R, SCHEME, 8, 32>();
    }
}

int stage_ctas_per_sm(const StageOpts& o) {
    if (o.precision == WM_PREC_MIXED) {
        switch (o.scheme) {
            case WM_SCHEME_KEP: return occupancy_tile<float, WM_SCHEME_KEP>(o.tile);
            case WM_SCHEME_MUSCL: return occupancy_tile<float, WM_SCHEME_MUSCL>(o.tile);
            default: return occupancy_tile<float, WM_SCHEME_HYBRID>(o.tile);
        }
    }
    switch (o.scheme) {
        case WM_SCHEME_KEP: return occupancy_tile<double, WM_SCHEME_KEP>(o.tile);
        case WM_SCHEME_MUSCL: return occupancy_tile<double, WM_SCHEME_MUSCL>(o.tile);
        default: return occupancy_tile<double, WM_SCHEME_HYBRID>(o.tile);
    }
}

cudaError_t launch_stage(const StageArgs& A, const StageOpts& o, cudaStream_t s) {
    if (o.precision == WM_PREC_MIXED) {
        switch (o.scheme) {
            case WM_SCHEME_KEP: return launch_tile<float, WM_SCHEME_KEP>(A, o, s);
            case WM_SCHEME_MUSCL: return launch_tile<float, WM_SCHEME_MUSCL>(A, o, s);
            default: return launch_tile<float, WM_SCHEME_HYBRID>(A, o, s);
        }
    }
    switch (o.scheme) {
        case WM_SCHEME_KEP: return launch_tile<double, WM_SCHEME_KEP>(A, o, s);
        case WM_SCHEME_MUSCL: return launch_tile<double, WM_SCHEME_MUSCL>(A, o, s);
        default: return launch_tile<double, WM_SCHEME_HYBRID>(A, o, s);
    }
}

void tile_shape(int tile, int* tj, int* tk) {
    switch (tile) {
        case 1: *tj = 16; *tk = 16; break;
        case 2: *tj = 4; *tk = 32; break;
        case 3: *tj = 16; *tk = 32; break;
        default: *tj = 8; *tk = 32; break;
    }
}

}  // namespace wm
