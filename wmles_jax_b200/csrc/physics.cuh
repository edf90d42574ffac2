// Per-cell and per-face physics of the wmles RHS, templated on the compute type R
// (double for the FP64 form, float for the mixed form).  Each function cites the
// reference formula it evaluates (EduardoMolina/wmles_jax).
#pragma once
#include <cuda_runtime.h>
#include "wm_internal.cuh"

namespace wm {

template <typename R>
struct Phys {
    R gamma, gm1, inv_gm1, Rg, inv_Rg, cp, inv_Pr, inv_Prt;
    R mu_ref, inv_Tref, TrefS, S_suth;
    R th0, inv_dth, sgs_c;
    __device__ explicit Phys(const CaseDev& c)
        : gamma(R(c.gamma)), gm1(R(c.gm1)), inv_gm1(R(c.inv_gm1)), Rg(R(c.Rg)), inv_Rg(R(c.inv_Rg)),
          cp(R(c.cp)), inv_Pr(R(c.inv_Pr)), inv_Prt(R(c.inv_Prt)), mu_ref(R(c.mu_ref)),
          inv_Tref(R(c.inv_Tref)), TrefS(R(c.TrefS)), S_suth(R(c.S_suth)), th0(R(c.th0)),
          inv_dth(R(c.inv_dth)), sgs_c(R(c.sgs_c)) {}
};

__device__ __forceinline__ double wm_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float wm_sqrt(float x) { return sqrtf(x); }

// primitive record kept per cell in shared memory: rho, u, v, w, p, T, e = p/((g-1)rho) + |u|^2/2
enum { PR_RHO = 0, PR_U, PR_V, PR_W, PR_P, PR_T, PR_E, PR_N };

// conservative -> primitive record, wmles/gas.py:28-33
template <typename R>
__device__ __forceinline__ void cons_to_rec(const double q[5], const Phys<R>& P, R out[PR_N]) {
    const R rho = R(q[0]);
    const R ir = R(1) / rho;
    const R u = R(q[1]) * ir, v = R(q[2]) * ir, w = R(q[3]) * ir;
    const R ke = R(0.5) * (u * u + v * v + w * w);
    const R p = P.gm1 * (R(q[4]) - rho * ke);
    out[PR_RHO] = rho; out[PR_U] = u; out[PR_V] = v; out[PR_W] = w; out[PR_P] = p;
    out[PR_T] = p * ir * P.inv_Rg;
    out[PR_E] = p * ir * P.inv_gm1 + ke;
}

// Sutherland viscosity, wmles/gas.py:24-26 ((T/T_ref)^1.5 as x sqrt(x))
template <typename R>
__device__ __forceinline__ R sutherland(R T, const Phys<R>& P) {
    const R x = T * P.inv_Tref;
    return P.mu_ref * (x * wm_sqrt(x)) * P.TrefS / (T + P.S_suth);
}

// Kennedy-Gruber two-point flux (already times the face area), wmles/schemes.py:15-23
template <typename R>
__device__ __forceinline__ void kg_flux(const R* a, const R* b, int s, R Sx, R Sy, R Sz, R F[5]) {
    const R rho = R(0.5) * (a[PR_RHO * s] + b[PR_RHO * s]);
    const R u = R(0.5) * (a[PR_U * s] + b[PR_U * s]);
    const R v = R(0.5) * (a[PR_V * s] + b[PR_V * s]);
    const R w = R(0.5) * (a[PR_W * s] + b[PR_W * s]);
    const R p = R(0.5) * (a[PR_P * s] + b[PR_P * s]);
    const R ea = R(0.5) * (a[PR_E * s] + b[PR_E * s]);
    const R un = u * Sx + v * Sy + w * Sz;
    const R m = rho * un;
    F[0] = m;
    F[1] = m * u + p * Sx;
    F[2] = m * v + p * Sy;
    F[3] = m * w + p * Sz;
    F[4] = m * ea + p * un;
}

// KEP order 2 / 4, wmles/schemes.py:57-70: 2 [(2/3) F(L,R) - (1/12) (F(L,R2) + F(L2,R))],
// written (4/3) F(L,R) - (1/6) (...) (the outer factor 2 moved into the constants: exact)
template <typename R>
__device__ __forceinline__ void kep_flux(int order, const R* L2, const R* L, const R* Rr, const R* R2,
                                         int s, R Sx, R Sy, R Sz, R F[5]) {
    kg_flux(L, Rr, s, Sx, Sy, Sz, F);
    if (order == 4) {
        R Fa[5], Fb[5];
        kg_flux(L, R2, s, Sx, Sy, Sz, Fa);
        kg_flux(L2, Rr, s, Sx, Sy, Sz, Fb);
#pragma unroll
        for (int v = 0; v < 5; ++v)
            F[v] = R(4.0 / 3.0) * F[v] - R(1.0 / 6.0) * (Fa[v] + Fb[v]);
    }
}

// limiters, wmles/schemes.py:100-105
template <typename R>
__device__ __forceinline__ R albada(R a, R b) {
    const R eps = R(1e-12);
    return (a * (b * b + eps) + b * (a * a + eps)) / (a * a + b * b + R(2) * eps);
}
template <typename R>
__device__ __forceinline__ R sgn(R a) { return R((a > R(0)) - (a < R(0))); }
template <typename R>
__device__ __forceinline__ R minmod(R a, R b) {
    return R(0.5) * (sgn(a) + sgn(b)) * fmin(fabs(a), fabs(b));
}

// HLLC flux times |S|, wmles/schemes.py:108-137
template <typename R>
__device__ __forceinline__ void hllc_flux(const R wl[5], const R wr[5], R Sx, R Sy, R Sz, R gamma,
                                          R inv_gm1, R F[5]) {
    const R Sm = wm_sqrt(Sx * Sx + Sy * Sy + Sz * Sz);
    const R iS = R(1) / Sm;
    const R nx = Sx * iS, ny = Sy * iS, nz = Sz * iS;
    const R rl = wl[0], ul = wl[1], vl = wl[2], wlz = wl[3], pl = wl[4];
    const R rr = wr[0], ur = wr[1], vr = wr[2], wrz = wr[3], pr = wr[4];
    const R unl = ul * nx + vl * ny + wlz * nz;
    const R unr = ur * nx + vr * ny + wrz * nz;
    const R cl = wm_sqrt(gamma * pl / rl), cr = wm_sqrt(gamma * pr / rr);
    const R sL = fmin(unl - cl, unr - cr), sR = fmax(unl + cl, unr + cr);
    const R ss = (pr - pl + rl * unl * (sL - unl) - rr * unr * (sR - unr)) /
                 (rl * (sL - unl) - rr * (sR - unr));
    // choose the side, then evaluate only that branch
    const bool left = (sL >= R(0)) || (ss >= R(0));
    const R r = left ? rl : rr, u = left ? ul : ur, v = left ? vl : vr, w = left ? wlz : wrz;
    const R p = left ? pl : pr, un = left ? unl : unr;
    const R E = p * inv_gm1 + R(0.5) * r * (u * u + v * v + w * w);
    R Fp[5];
    Fp[0] = r * un;
    Fp[1] = r * un * u + p * nx;
    Fp[2] = r * un * v + p * ny;
    Fp[3] = r * un * w + p * nz;
    Fp[4] = (E + p) * un;
    const bool star = left ? !(sL >= R(0)) : (sR > R(0));
    if (star) {
        const R s = left ? sL : sR;
        const R f = r * (s - un) / (s - ss);
        const R e = E / r + (ss - un) * (ss + p / (r * (s - un)));
        const R d = ss - un;
        Fp[0] += s * (f - r);
        Fp[1] += s * (f * (u + d * nx) - r * u);
        Fp[2] += s * (f * (v + d * ny) - r * v);
        Fp[3] += s * (f * (w + d * nz) - r * w);
        Fp[4] += s * (f * e - E);
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) F[q] = Fp[q] * Sm;
}

// MUSCL reconstruction with positivity fallback + HLLC, wmles/schemes.py:140-152
template <typename R>
__device__ __forceinline__ void muscl_hllc_flux(int limiter, const R* L2, const R* L, const R* Rr,
                                                const R* R2, int s, R Sx, R Sy, R Sz,
                                                const Phys<R>& P, R F[5]) {
    R wl[5], wr[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        const R a = L[v * s] - L2[v * s], b = Rr[v * s] - L[v * s], c = R2[v * s] - Rr[v * s];
        if (limiter == WM_LIMITER_MINMOD) {
            wl[v] = L[v * s] + R(0.5) * minmod(a, b);
            wr[v] = Rr[v * s] - R(0.5) * minmod(b, c);
        } else {
            wl[v] = L[v * s] + R(0.5) * albada(a, b);
            wr[v] = Rr[v * s] - R(0.5) * albada(b, c);
        }
    }
    if (wl[0] <= R(0) || wl[4] <= R(0) || wr[0] <= R(0) || wr[4] <= R(0)) {
#pragma unroll
        for (int v = 0; v < 5; ++v) { wl[v] = L[v * s]; wr[v] = Rr[v * s]; }
    }
    hllc_flux(wl, wr, Sx, Sy, Sz, P.gamma, P.inv_gm1, F);
}

// SGS eddy viscosity nu_t from g[i][j] = du_i/dx_j, wmles/sgs.py:14-42
template <typename R>
__device__ __forceinline__ R sgs_nut(int model, const R g[9], R delta, R c) {
    if (model == WM_SGS_SMAGORINSKY) {
        R ss = R(0);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const R s = R(0.5) * (g[3 * i + j] + g[3 * j + i]);
                ss += s * s;
            }
        const R cd = c * delta;
        return cd * cd * wm_sqrt(R(2) * ss);
    }
    if (model == WM_SGS_WALE) {
        // S_ij S_ij and S^d_ij S^d_ij from the six distinct entries of each symmetric tensor
        // (off-diagonal squares counted twice, an exact doubling), summed as trees: the
        // reference's contractions up to the order of the additions, with dependency chains
        // of four additions instead of nine
        R g2[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                g2[3 * i + j] = g[3 * i] * g[j] + g[3 * i + 1] * g[3 + j] + g[3 * i + 2] * g[6 + j];
        const R s01 = R(0.5) * (g[1] + g[3]), s02 = R(0.5) * (g[2] + g[6]), s12 = R(0.5) * (g[5] + g[7]);
        const R ss = ((g[0] * g[0] + g[4] * g[4]) + g[8] * g[8]) + R(2) * ((s01 * s01 + s02 * s02) + s12 * s12);
        const R tr = (g2[0] + g2[4] + g2[8]) * R(1.0 / 3.0);
        const R d0 = g2[0] - tr, d1 = g2[4] - tr, d2 = g2[8] - tr;
        const R q01 = R(0.5) * (g2[1] + g2[3]), q02 = R(0.5) * (g2[2] + g2[6]), q12 = R(0.5) * (g2[5] + g2[7]);
        const R sdsd = ((d0 * d0 + d1 * d1) + d2 * d2) + R(2) * ((q01 * q01 + q02 * q02) + q12 * q12);
        const R cd = c * delta;
        const R rsd = wm_sqrt(sdsd), rss = wm_sqrt(ss);
        return cd * cd * (sdsd * rsd) / (ss * ss * rss + sdsd * wm_sqrt(rsd) + R(1e-30));
    }
    if (model == WM_SGS_VREMAN) {
        const R d2 = delta * delta;
        R b[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                b[3 * i + j] = d2 * (g[3 * i] * g[3 * j] + g[3 * i + 1] * g[3 * j + 1] + g[3 * i + 2] * g[3 * j + 2]);
        const R Bb = b[0] * b[4] - b[1] * b[1] + b[0] * b[8] - b[2] * b[2] + b[4] * b[8] - b[5] * b[5];
        R aa = R(0);
#pragma unroll
        for (int i = 0; i < 9; ++i) aa += g[i] * g[i];
        return R(2.5) * c * c * wm_sqrt(fmax(Bb, R(0)) / (aa + R(1e-30)));
    }
    return R(0);
}

// Ducros sensor, wmles/viscous.py:22-25
template <typename R>
__device__ __forceinline__ R ducros(const R g[9]) {
    const R div = g[0] + g[4] + g[8];
    const R a = g[7] - g[5], b = g[2] - g[6], c = g[3] - g[1];
    const R w2 = a * a + b * b + c * c;
    return div * div / (div * div + w2 + R(1e-30));
}

// ------------------------------------------------------------------ wall model (FP64)
// Spalding's law solved for u+ by safeguarded Newton, wmles/wall_model.py:19-40
// *moving is set when the iteration ends with an update larger than 1e-8 of the iterate
// (not settled within n_iter; the reference returns that iterate all the same)
__device__ __forceinline__ double spalding_utau(double kappa, double ekb, int n_iter, double h, double U,
                                                double rho_w, double mu_w, bool* moving) {
    const double Reh = h * U * rho_w / mu_w;
    double up = fmin(fmax(sqrt(Reh), 1.0), 25.0);
    double last = 0.0, prev = up;
    *moving = false;
    for (int it = 0; it < n_iter; ++it) {
        const double ku = kappa * up;
        const double ex = exp(ku);
        const double F = up + ekb * (ex - 1.0 - ku - 0.5 * ku * ku - ku * ku * ku / 6.0) - Reh / up;
        const double dF = 1.0 + ekb * kappa * (ex - 1.0 - ku - 0.5 * ku * ku) + Reh / (up * up);
        const double next = fmin(fmax(up - F / dF, 0.5 * up), 100.0);
        // the update is a fixed function of up: once an iterate repeats exactly, every later
        // one does too, so stopping here returns what all n_iter iterations would
        if (next == up) return U / up;
        // period two (about one face in ten ends alternating between two neighbouring
        // doubles, and one such lane kept its whole warp iterating to n_iter): the iterates
        // from prev on are prev, up, prev, ..., so the last of n_iter is prev (= next) when
        // n_iter - (it - 1) is even, else up
        if (it > 0 && next == prev) {
            const double fin = ((n_iter - it + 1) & 1) == 0 ? next : up;
            *moving = !(fabs(next - up) <= 1e-8 * fin);
            return U / fin;
        }
        last = next - up;
        prev = up;
        up = next;
    }
    *moving = !(fabs(last) <= 1e-8 * up);
    return U / up;
}

}  // namespace wm
