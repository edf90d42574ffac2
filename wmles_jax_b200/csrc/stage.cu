// Fused RHS + SSP-RK3 stage kernel.
//
// One CTA owns a TJ x TK tile of (j,k) columns of one block and marches along i over a
// chunk of planes [i0, i1).  Per plane it keeps, in shared memory:
//   pr[4]  primitive records of planes i-2..i+1 on the tile + 2-cell halo (rolling ring)
//   gs     Green-Gauss gradients, mu_eff, k_eff (and the Ducros sensor) of plane i on the
//          tile + 1-cell halo
//   fj/fk  the j- and k-face fluxes of plane i
// and in registers, per column, the i-face flux of the previous face, the j/k flux
// differences of the previous plane and that plane's gradient record.  Each face flux is
// evaluated once; each conservative value is read from HBM about once per stage (halo
// re-reads hit L2).  The epilogue combines the flux divergence with the RK stage and
// writes the new state; stage 3 also emits per-tile partial sums of rho u V for the
// constant-mass-flux constraint.
//
// Reference: Solver._block_rhs (wmles/solver.py:76-95), green_gauss / viscous_flux /
// ducros (wmles/viscous.py), schemes (wmles/schemes.py), SGS (wmles/sgs.py), SSP-RK3
// (wmles/solver.py:110-121).
#include <cstdio>
#include "physics.cuh"
#include "stage.cuh"

namespace wm {

template <typename R, int SCHEME, int TJ, int TK>
struct StageLayout {
    static constexpr int NT = TJ * TK;
    static constexpr int PJ = TJ + 4, PK = TK + 4, PN = PJ * PK;   // primitives: 2-cell halo
    static constexpr int GJ = TJ + 2, GK = TK + 2, GN = GJ * GK;   // gradients: 1-cell halo
    static constexpr int NGS = (SCHEME == WM_SCHEME_HYBRID) ? 15 : 14;
    static constexpr int FJN = (TJ + 1) * TK, FKN = TJ * (TK + 1);
    static constexpr size_t body = sizeof(R) * (size_t(4) * PR_N * PN + size_t(NGS) * GN + 5 * (FJN + FKN));
    static constexpr size_t red_off = (body + 15) / 16 * 16;        // reduction scratch, 16-byte aligned
    static constexpr size_t bytes = red_off + sizeof(double) * 32;
};

// gradient record: g[0..11] = d(u,v,w,T)/d(x,y,z), 12 = mu_eff, 13 = k_eff, 14 = theta
enum { GS_MU = 12, GS_K = 13, GS_TH = 14 };

template <typename R>
__device__ __forceinline__ R met(const BlockDev& B, int comp, long long idx) {
    if constexpr (sizeof(R) == 4) return __ldg(B.met32 + comp * B.ncell + idx);
    else return __ldg(B.met + comp * B.ncell + idx);
}

// centroid difference xc[idx] - xc[idx - off] from the FP64 coordinates (in the mixed form
// too: a float difference of nearby large coordinates would lose the spacing)
template <typename R>
__device__ __forceinline__ R xdiff(const BlockDev& B, int comp, long long idx, long long off) {
    const double* x = B.met + comp * B.ncell;
    return R(__ldg(x + idx) - __ldg(x + idx - off));
}

// viscous flux through one face (times area), wmles/viscous.py:28-51.  gL/gR index a
// gradient record; pl/pr point at primitive records with component stride s.
template <typename R, class GL, class GR>
__device__ __forceinline__ void viscous_flux(const R* pl, const R* pr, int s, GL gL, GR gR, R Sx, R Sy, R Sz,
                                             R dx, R dy, R dz, R F[5]) {
    const R dist = wm_sqrt(dx * dx + dy * dy + dz * dz);
    const R idist = R(1) / dist;
    const R e0 = dx * idist, e1 = dy * idist, e2 = dz * idist;
    R gf[12];
    const int pv[4] = {PR_U, PR_V, PR_W, PR_T};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const R b0 = R(0.5) * (gL(3 * a) + gR(3 * a));
        const R b1 = R(0.5) * (gL(3 * a + 1) + gR(3 * a + 1));
        const R b2 = R(0.5) * (gL(3 * a + 2) + gR(3 * a + 2));
        const R corr = (pr[pv[a] * s] - pl[pv[a] * s]) * idist - (b0 * e0 + b1 * e1 + b2 * e2);
        gf[3 * a] = b0 + corr * e0;
        gf[3 * a + 1] = b1 + corr * e1;
        gf[3 * a + 2] = b2 + corr * e2;
    }
    const R div = gf[0] + gf[4] + gf[8];
    const R muf = R(0.5) * (gL(GS_MU) + gR(GS_MU));
    const R kf = R(0.5) * (gL(GS_K) + gR(GS_K));
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

// total face flux (inviscid scheme + viscous), S = face area vector, d = xc_R - xc_L
template <typename R, int SCHEME, class GL, class GR>
__device__ __forceinline__ void face_flux(const StageOpts& o, const Phys<R>& P, const R* L2, const R* L,
                                          const R* Rr, const R* R2, int s, GL gL, GR gR, R Sx, R Sy,
                                          R Sz, R dx, R dy, R dz, R F[5]) {
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
    viscous_flux<R>(L, Rr, s, gL, gR, Sx, Sy, Sz, dx, dy, dz, F);
}

template <typename R, int SCHEME, int TJ, int TK>
__global__ void __launch_bounds__(TJ* TK, 1) stage_kernel(const __grid_constant__ StageArgs A, const StageOpts o) {
    using LY = StageLayout<R, SCHEME, TJ, TK>;
    constexpr int NT = LY::NT, PK = LY::PK, PN = LY::PN, GK = LY::GK, GN = LY::GN, NGS = LY::NGS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* pr = reinterpret_cast<R*>(smem_raw);                 // [4][PR_N][PN]
    R* gs = pr + 4 * PR_N * PN;                             // [NGS][GN]
    R* fj = gs + NGS * GN;                                  // [5][FJN]
    R* fk = fj + 5 * LY::FJN;                               // [5][FKN]
    double* red = reinterpret_cast<double*>(smem_raw + LY::red_off);

    const Tile t = A.tiles[blockIdx.x];
    const BlockDev B = A.blocks[t.blk];
    const CaseDev& C = A.cases[B.case_id];
    const Phys<R> P(C);
    const StatePtrs SP = A.p[t.blk];
    const int ng = B.ng, Nj = B.N[1], Nk = B.N[2];
    const long long plane = B.plane, ncell = B.ncell;
    const int tid = threadIdx.x, tj = tid / TK, tk = tid % TK;
    const int jhi = ng + B.n[1], khi = ng + B.n[2], ihi = ng + B.n[0];
    const int j = t.j0 + tj, k = t.k0 + tk;
    const bool active = (j < jhi) && (k < khi);
    const int sgs_model = o.sgs;

    // ---- load plane ip into ring slot: primitive records on the tile + 2-cell halo
    auto load_plane = [&](int ip, int slot) {
        R* dst = pr + slot * PR_N * PN;
        for (int c = tid; c < PN; c += NT) {
            const int jj = c / PK, kk = c - jj * PK;
            const int gj = min(max(t.j0 - 2 + jj, 0), Nj - 1);
            const int gk = min(max(t.k0 - 2 + kk, 0), Nk - 1);
            const long long idx = ip * plane + (long long)gj * Nk + gk;
            double q[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) q[v] = __ldg(SP.q_in + v * ncell + idx);
            R rec[PR_N];
            cons_to_rec(q, P, rec);
#pragma unroll
            for (int v = 0; v < PR_N; ++v) dst[v * PN + c] = rec[v];
        }
    };

    // ---- gradient records of plane ip (ring slots of ip-1, ip, ip+1) on the tile + 1-cell halo
    auto grad_plane = [&](int ip, int sm, int s0, int sp) {
        const R* Pm = pr + sm * PR_N * PN;
        const R* P0 = pr + s0 * PR_N * PN;
        const R* Pp = pr + sp * PR_N * PN;
        for (int c = tid; c < GN; c += NT) {
            const int jj = c / GK, kk = c - jj * GK;
            const int pc = (jj + 1) * PK + (kk + 1);
            const int gj = min(t.j0 - 1 + jj, Nj - 2), gk = min(t.k0 - 1 + kk, Nk - 2);
            const long long idx = ip * plane + (long long)gj * Nk + gk;
            const int pv[4] = {PR_U, PR_V, PR_W, PR_T};
            R acc[12];
#pragma unroll
            for (int q = 0; q < 12; ++q) acc[q] = R(0);
            // direction 0 (i): neighbours in the ring
            {
                const R Slx = met<R>(B, WM_MET_SIX, idx), Sly = met<R>(B, WM_MET_SIY, idx), Slz = met<R>(B, WM_MET_SIZ, idx);
                const R Shx = met<R>(B, WM_MET_SIX, idx + plane), Shy = met<R>(B, WM_MET_SIY, idx + plane),
                        Shz = met<R>(B, WM_MET_SIZ, idx + plane);
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const R c0 = P0[pv[a] * PN + pc];
                    const R lo = R(0.5) * (Pm[pv[a] * PN + pc] + c0), hi = R(0.5) * (c0 + Pp[pv[a] * PN + pc]);
                    acc[3 * a] += hi * Shx - lo * Slx;
                    acc[3 * a + 1] += hi * Shy - lo * Sly;
                    acc[3 * a + 2] += hi * Shz - lo * Slz;
                }
            }
            // direction 1 (j)
            {
                const R Slx = met<R>(B, WM_MET_SJX, idx), Sly = met<R>(B, WM_MET_SJY, idx), Slz = met<R>(B, WM_MET_SJZ, idx);
                const R Shx = met<R>(B, WM_MET_SJX, idx + Nk), Shy = met<R>(B, WM_MET_SJY, idx + Nk),
                        Shz = met<R>(B, WM_MET_SJZ, idx + Nk);
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const R c0 = P0[pv[a] * PN + pc];
                    const R lo = R(0.5) * (P0[pv[a] * PN + pc - PK] + c0), hi = R(0.5) * (c0 + P0[pv[a] * PN + pc + PK]);
                    acc[3 * a] += hi * Shx - lo * Slx;
                    acc[3 * a + 1] += hi * Shy - lo * Sly;
                    acc[3 * a + 2] += hi * Shz - lo * Slz;
                }
            }
            // direction 2 (k)
            {
                const R Slx = met<R>(B, WM_MET_SKX, idx), Sly = met<R>(B, WM_MET_SKY, idx), Slz = met<R>(B, WM_MET_SKZ, idx);
                const R Shx = met<R>(B, WM_MET_SKX, idx + 1), Shy = met<R>(B, WM_MET_SKY, idx + 1),
                        Shz = met<R>(B, WM_MET_SKZ, idx + 1);
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const R c0 = P0[pv[a] * PN + pc];
                    const R lo = R(0.5) * (P0[pv[a] * PN + pc - 1] + c0), hi = R(0.5) * (c0 + P0[pv[a] * PN + pc + 1]);
                    acc[3 * a] += hi * Shx - lo * Slx;
                    acc[3 * a + 1] += hi * Shy - lo * Sly;
                    acc[3 * a + 2] += hi * Shz - lo * Slz;
                }
            }
            const R ivol = R(1) / met<R>(B, WM_MET_VOL, idx);
#pragma unroll
            for (int q = 0; q < 12; ++q) acc[q] *= ivol;
            const R T = P0[PR_T * PN + pc];
            const R mu = sutherland(T, P);
            R mut = R(0);
            if (sgs_model != WM_SGS_NONE)
                mut = P0[PR_RHO * PN + pc] * sgs_nut(sgs_model, acc, met<R>(B, WM_MET_DELTA, idx), P.sgs_c);
#pragma unroll
            for (int q = 0; q < 12; ++q) gs[q * GN + c] = acc[q];
            gs[GS_MU * GN + c] = mu + mut;
            gs[GS_K * GN + c] = P.cp * (mu * P.inv_Pr + mut * P.inv_Prt);
            if constexpr (NGS > 14) gs[GS_TH * GN + c] = ducros(acc);
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
    auto iface_flux = [&](int ip, R F[5]) {
        if (ip == ng && wall_flux(0, j, k, F)) return;
        if (ip == ihi && wall_flux(1, j, k, F)) return;
        const int pc = (tj + 2) * PK + (tk + 2);
        const int gc = (tj + 1) * GK + (tk + 1);
        const R* L2 = pr + ((ip - 2) & 3) * PR_N * PN + pc;
        const R* L = pr + ((ip - 1) & 3) * PR_N * PN + pc;
        const R* Rr = pr + (ip & 3) * PR_N * PN + pc;
        const R* R2 = pr + ((ip + 1) & 3) * PR_N * PN + pc;
        const long long idx = ip * plane + (long long)j * Nk + k;
        const R Sx = met<R>(B, WM_MET_SIX, idx), Sy = met<R>(B, WM_MET_SIY, idx), Sz = met<R>(B, WM_MET_SIZ, idx);
        const R dx = xdiff<R>(B, WM_MET_XCX, idx, plane);
        const R dy = xdiff<R>(B, WM_MET_XCY, idx, plane);
        const R dz = xdiff<R>(B, WM_MET_XCZ, idx, plane);
        face_flux<R, SCHEME>(o, P, L2, L, Rr, R2, PN, [&](int v) { return gsp[v]; },
                             [&](int v) { return gs[v * GN + gc]; }, Sx, Sy, Sz, dx, dy, dz, F);
    };

    // ---- j- and k-face fluxes of plane ip into shared memory
    auto jk_fluxes = [&](int ip) {
        const R* P0 = pr + (ip & 3) * PR_N * PN;
        for (int f = tid; f < LY::FJN; f += NT) {
            const int row = f / TK, kk = f - row * TK;
            const int gj = t.j0 + row, gk = t.k0 + kk;
            R F[5] = {R(0), R(0), R(0), R(0), R(0)};
            if (gj <= jhi && gk < khi) {
                bool done = false;
                if (gj == ng) done = wall_flux(2, ip, gk, F);
                else if (gj == jhi) done = wall_flux(3, ip, gk, F);
                if (!done) {
                    const int pc = (row + 2) * PK + (kk + 2);     // R cell in the primitive tile
                    const int gc = (row + 1) * GK + (kk + 1);     // R cell in the gradient tile
                    const long long idx = ip * plane + (long long)gj * Nk + gk;
                    const R Sx = met<R>(B, WM_MET_SJX, idx), Sy = met<R>(B, WM_MET_SJY, idx), Sz = met<R>(B, WM_MET_SJZ, idx);
                    const R dx = xdiff<R>(B, WM_MET_XCX, idx, Nk);
                    const R dy = xdiff<R>(B, WM_MET_XCY, idx, Nk);
                    const R dz = xdiff<R>(B, WM_MET_XCZ, idx, Nk);
                    face_flux<R, SCHEME>(o, P, P0 + pc - 2 * PK, P0 + pc - PK, P0 + pc, P0 + pc + PK, PN,
                                         [&](int v) { return gs[v * GN + gc - GK]; },
                                         [&](int v) { return gs[v * GN + gc]; }, Sx, Sy, Sz, dx, dy, dz, F);
                }
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) fj[v * LY::FJN + f] = F[v];
        }
        for (int f = tid; f < LY::FKN; f += NT) {
            const int row = f / (TK + 1), col = f - row * (TK + 1);
            const int gj = t.j0 + row, gk = t.k0 + col;
            R F[5] = {R(0), R(0), R(0), R(0), R(0)};
            if (gj < jhi && gk <= khi) {
                bool done = false;
                if (gk == ng) done = wall_flux(4, ip, gj, F);
                else if (gk == khi) done = wall_flux(5, ip, gj, F);
                if (!done) {
                    const int pc = (row + 2) * PK + (col + 2);
                    const int gc = (row + 1) * GK + (col + 1);
                    const long long idx = ip * plane + (long long)gj * Nk + gk;
                    const R Sx = met<R>(B, WM_MET_SKX, idx), Sy = met<R>(B, WM_MET_SKY, idx), Sz = met<R>(B, WM_MET_SKZ, idx);
                    const R dx = xdiff<R>(B, WM_MET_XCX, idx, 1);
                    const R dy = xdiff<R>(B, WM_MET_XCY, idx, 1);
                    const R dz = xdiff<R>(B, WM_MET_XCZ, idx, 1);
                    face_flux<R, SCHEME>(o, P, P0 + pc - 2, P0 + pc - 1, P0 + pc, P0 + pc + 1, PN,
                                         [&](int v) { return gs[v * GN + gc - 1]; },
                                         [&](int v) { return gs[v * GN + gc]; }, Sx, Sy, Sz, dx, dy, dz, F);
                }
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) fk[v * LY::FKN + f] = F[v];
        }
    };

    auto save_gs = [&]() {
        const int gc = (tj + 1) * GK + (tk + 1);
#pragma unroll
        for (int v = 0; v < NGS; ++v) gsp[v] = gs[v * GN + gc];
    };

    R dFj[5], dFk[5], Flo[5];
    auto jk_diff = [&]() {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            dFj[v] = fj[v * LY::FJN + (tj + 1) * TK + tk] - fj[v * LY::FJN + tj * TK + tk];
            dFk[v] = fk[v * LY::FKN + tj * (TK + 1) + tk + 1] - fk[v * LY::FKN + tj * (TK + 1) + tk];
        }
    };

    const int i0 = t.i0, i1 = t.i1;
    const double dt = A.stage ? A.dt[B.case_id] : 0.0;
    double cmf_acc = 0.0;

    // ---- prologue: planes i0-2 .. i0+1, gradients of i0-1 and i0, faces of plane i0
    load_plane(i0 - 2, (i0 - 2) & 3);
    load_plane(i0 - 1, (i0 - 1) & 3);
    load_plane(i0, i0 & 3);
    load_plane(i0 + 1, (i0 + 1) & 3);
    __syncthreads();
    // plane i0-1 needs plane i0-2's ring slot as its lower neighbour
    grad_plane(i0 - 1, (i0 - 2) & 3, (i0 - 1) & 3, i0 & 3);
    __syncthreads();
    save_gs();
    __syncthreads();
    grad_plane(i0, (i0 - 1) & 3, i0 & 3, (i0 + 1) & 3);
    __syncthreads();
    if (active) iface_flux(i0, Flo);
    jk_fluxes(i0);
    __syncthreads();
    jk_diff();
    save_gs();
    __syncthreads();

    // ---- march: iteration ip outputs plane ip-1
    for (int ip = i0 + 1; ip <= i1; ++ip) {
        load_plane(ip + 1, (ip + 1) & 3);
        __syncthreads();
        grad_plane(ip, (ip - 1) & 3, ip & 3, (ip + 1) & 3);
        __syncthreads();
        R Fhi[5];
        if (active) iface_flux(ip, Fhi);
        if (ip < i1) jk_fluxes(ip);
        if (active) {
            const int io = ip - 1;
            const long long idx = io * plane + (long long)j * Nk + k;
            const R ivol = R(1) / met<R>(B, WM_MET_VOL, idx);
            R r[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) r[v] = ((-(Fhi[v] - Flo[v]) - dFj[v]) - dFk[v]) * ivol;
            double rq[5], qi[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) qi[v] = __ldg(SP.q_in + v * ncell + idx);
            if (C.sponge) {
                // -sigma(x) (q - spanwise mean), wmles/smooth_ramp.py:212-221
                const double xl = __ldg(B.met + WM_MET_XCX * ncell + idx) * C.sp_invL;
                const double eta = fmin(fmax((xl - C.sp_xs) * C.sp_inv_dx, 0.0), 1.0);
                const double sig = C.sp_sigma0 * (eta * eta * eta * (10.0 + eta * (-15.0 + 6.0 * eta)));
                const long long mi = (long long)io * Nj + j;
                const long long mn = (long long)B.N[0] * Nj;
#pragma unroll
                for (int v = 0; v < 5; ++v) rq[v] = double(r[v]) - sig * (qi[v] - SP.spmean[v * mn + mi]);
            } else {
#pragma unroll
                for (int v = 0; v < 5; ++v) rq[v] = double(r[v]);
            }
            if (A.stage == 0) {
#pragma unroll
                for (int v = 0; v < 5; ++v) SP.q_out[v * ncell + idx] = rq[v];
            } else if (A.stage == 1) {
#pragma unroll
                for (int v = 0; v < 5; ++v) SP.q_out[v * ncell + idx] = qi[v] + dt * rq[v];
            } else if (A.stage == 2) {
#pragma unroll
                for (int v = 0; v < 5; ++v)
                    SP.q_out[v * ncell + idx] = 0.75 * __ldg(SP.q0 + v * ncell + idx) + 0.25 * (qi[v] + dt * rq[v]);
            } else {
                double qn[5];
#pragma unroll
                for (int v = 0; v < 5; ++v) {
                    qn[v] = (1.0 / 3.0) * __ldg(SP.q0 + v * ncell + idx) + (2.0 / 3.0) * (qi[v] + dt * rq[v]);
                    SP.q_out[v * ncell + idx] = qn[v];
                }
                if (C.cmf_dir >= 0) cmf_acc += qn[1 + C.cmf_dir] * __ldg(B.met + WM_MET_VOL * ncell + idx);
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) Flo[v] = Fhi[v];
        }
        __syncthreads();
        if (ip < i1) {
            jk_diff();
            save_gs();
        }
        __syncthreads();
    }

    if (A.stage == 3 && A.cmf_part != nullptr) {
        // fixed-order block reduction -> one partial per tile
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) cmf_acc += __shfl_down_sync(0xffffffffu, cmf_acc, off);
        if ((tid & 31) == 0) red[tid >> 5] = cmf_acc;
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < NT / 32; ++w) s += red[w];
            A.cmf_part[blockIdx.x] = s;
        }
    }
}

template <typename R, int SCHEME, int TJ, int TK>
static cudaError_t launch_one(const StageArgs& A, const StageOpts& o, cudaStream_t s) {
    using LY = StageLayout<R, SCHEME, TJ, TK>;
    auto kern = stage_kernel<R, SCHEME, TJ, TK>;
    static bool configured = false;   // per instantiation; device attribute set once per process
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LY::bytes);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    kern<<<A.ntiles, LY::NT, LY::bytes, s>>>(A, o);
    return cudaGetLastError();
}

template <typename R, int SCHEME, int TJ, int TK>
static int occupancy_one() {
    using LY = StageLayout<R, SCHEME, TJ, TK>;
    auto kern = stage_kernel<R, SCHEME, TJ, TK>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LY::bytes) != cudaSuccess) return 1;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, LY::NT, LY::bytes) != cudaSuccess) return 1;
    return n;
}

template <typename R, int SCHEME>
static int occupancy_tile(int tile) {
    switch (tile) {
        case 1: return occupancy_one<R, SCHEME, 16, 16>();
        case 2: return occupancy_one<R, SCHEME, 4, 32>();
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

template <typename R, int SCHEME>
static cudaError_t launch_tile(const StageArgs& A, const StageOpts& o, cudaStream_t s) {
    switch (o.tile) {
        case 1: return launch_one<R, SCHEME, 16, 16>(A, o, s);
        case 2: return launch_one<R, SCHEME, 4, 32>(A, o, s);
        default: return launch_one<R, SCHEME, 8, 32>(A, o, s);
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
        default: *tj = 8; *tk = 32; break;
    }
}

size_t stage_smem_bytes(int precision, int scheme, int tile) {
    int tj, tk;
    tile_shape(tile, &tj, &tk);
    const size_t rs = precision == WM_PREC_MIXED ? 4 : 8;
    const int ngs = scheme == WM_SCHEME_HYBRID ? 15 : 14;
    const size_t body = rs * (size_t(4) * PR_N * (tj + 4) * (tk + 4) + size_t(ngs) * (tj + 2) * (tk + 2) +
                              5 * ((tj + 1) * tk + tj * (tk + 1)));
    return (body + 15) / 16 * 16 + sizeof(double) * 32;
}

}  // namespace wm
