// Surface kernels of the step: the ghost-cell gather, the wall model and the sponge means.
//
// Ghost cells: the host traces the reference's ghost-fill order (Solver.apply_bcs,
// wmles/solver.py:59-73: passes x axes x blocks x sides of block-to-block exchange or BC
// mirror fill) on cell indices, so every ghost cell becomes "take one source value (an
// interior cell of some block, a synthetic-inflow value or a constant state) and apply a
// short chain of per-cell maps".  The maps are the reference's BC maps (wmles/bc.py:41-115)
// evaluated in the same FP64 operation order as NumPy; this file is compiled with
// -fmad=false so no multiply-add is contracted, which makes the gather bit-identical to the
// reference's ghost fill (and keeps the wall model and the sponge means, which share the
// file, in NumPy's rounding as well).
//
// Before every stage kernel one launch (surface_kernel) does all three: the parts read
// disjoint data (ghost cells are written; the wall model and the sponge means read interior
// cells only), so they overlap instead of running as three dependent launches.
#include "wm_internal.cuh"
#include "physics.cuh"
#include "aux.cuh"

namespace wm {

// q -> (rho, u, v, w, p), T ; wmles/gas.py:28-33
__device__ __forceinline__ void g_c2p(const double q[5], double gm1, double Rg, double w[5], double& T) {
    const double rho = q[0];
    const double u = q[1] / rho, v = q[2] / rho, ww = q[3] / rho;
    const double ke = (u * u + v * v) + ww * ww;
    const double p = gm1 * (q[4] - (0.5 * rho) * ke);
    w[0] = rho; w[1] = u; w[2] = v; w[3] = ww; w[4] = p;
    T = p / (rho * Rg);
}

// (rho, u, v, w, p) -> q ; wmles/gas.py:35-38
__device__ __forceinline__ void g_p2c(const double w[5], double gm1, double q[5]) {
    const double ke = (w[1] * w[1] + w[2] * w[2]) + w[3] * w[3];
    q[0] = w[0];
    q[1] = w[0] * w[1];
    q[2] = w[0] * w[2];
    q[3] = w[0] * w[3];
    q[4] = w[4] / gm1 + (0.5 * w[0]) * ke;
}

__device__ __forceinline__ void op_slip(double q[5], const double n[3], double gm1, double Rg) {
    // wmles/bc.py:41-47
    double w[5], T;
    g_c2p(q, gm1, Rg, w, T);
    const double un = (w[1] * n[0] + w[2] * n[1]) + w[3] * n[2];
    const double t = 2.0 * un;
    w[1] = w[1] - t * n[0];
    w[2] = w[2] - t * n[1];
    w[3] = w[3] - t * n[2];
    g_p2c(w, gm1, q);
}

__device__ __forceinline__ void op_noslip(double q[5], const double* bc, double gm1, double Rg) {
    // wmles/bc.py:56-64 ; bc[5] = T_wall, bc[6] = isothermal flag
    double w[5], T;
    g_c2p(q, gm1, Rg, w, T);
    double Tg = T;
    if (bc[6] != 0.0) {
        const double a = 2.0 * bc[5] - T, b = 0.1 * bc[5];
        Tg = (a > b || a != a) ? a : b;      // np.maximum (propagates NaN)
    }
    w[0] = w[4] / (Rg * Tg);
    w[1] = -w[1]; w[2] = -w[2]; w[3] = -w[3];
    g_p2c(w, gm1, q);
}

__device__ __forceinline__ void op_farfield(double q[5], const double nrm[3], int side, const double* bc,
                                            double gamma, double gm1, double Rg) {
    // linearised characteristics, wmles/bc.py:86-115 ; bc[0..4] = prim_inf
    double w[5], T;
    g_c2p(q, gm1, Rg, w, T);
    const double ri = bc[0], ui[3] = {bc[1], bc[2], bc[3]}, pi = bc[4];
    const double ci = sqrt(gamma * pi / ri);
    const double n[3] = {side ? nrm[0] : -nrm[0], side ? nrm[1] : -nrm[1], side ? nrm[2] : -nrm[2]};
    const double un = (w[1] * n[0] + w[2] * n[1]) + w[3] * n[2];
    const double uni = (ui[0] * n[0] + ui[1] * n[1]) + ui[2] * n[2];
    const double c = sqrt((gamma * Rg) * T);
    const double drho = w[0] - ri, dp = w[4] - pi, dun = un - uni;
    const double rc = ri * ci;
    const double ap = (un + c > 0.0) ? dp + rc * dun : 0.0;
    const double am = (un - c > 0.0) ? dp - rc * dun : 0.0;
    const double dp_bc = 0.5 * (ap + am);
    const double dun_bc = (ap - am) / ((2.0 * ri) * ci);
    const bool out = un > 0.0;
    const double ci2 = ci * ci;
    const double ent = out ? drho - dp / ci2 : 0.0;
    double o[5];
    o[0] = (ri + dp_bc / ci2) + ent;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double dut = out ? (w[1 + a] - ui[a]) - dun * n[a] : 0.0;
        o[1 + a] = (ui[a] + dun_bc * n[a]) + dut;
    }
    o[4] = pi + dp_bc;
    g_p2c(o, gm1, q);
}

// segment (case) holding launch entry e: segments are in entry order
__device__ __forceinline__ int find_seg(const GhostArgs& G, int e) {
    int lo = 0, hi = G.nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (G.segs[mid].start <= e) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ghost entry e of the launch: gather its source value and apply its map chain; the value
// goes to the destination ghost cell, or to the stash in two-phase mode
__device__ __forceinline__ void ghost_entry(const GhostArgs& G, int e) {
    const GhostSeg& S = G.segs[find_seg(G, e)];
    const int le = e - S.start;
    const int sk = S.src[2 * le], sc = S.src[2 * le + 1];
    const int kind = sk >> 24, sb = sk & 0xffffff;
    double q[5];
    if (kind == WM_SRC_CELL) {
        const double* s = G.q[S.block0 + sb];
        const long long n = G.ncell[S.block0 + sb];
#pragma unroll
        for (int v = 0; v < 5; ++v) q[v] = s[v * n + sc];
    } else if (kind == WM_SRC_INFLOW) {
#pragma unroll
        for (int v = 0; v < 5; ++v) q[v] = S.inflow[v * S.inflow_n + sc];
    } else {
#pragma unroll
        for (int v = 0; v < 5; ++v) q[v] = S.bc[8 * sb + v];
    }
    const int o0 = S.ops[2 * le], no = S.ops[2 * le + 1];
    for (int i = 0; i < no; ++i) {
        const int code = S.op_code[o0 + i];
        const double* nrm = S.op_nrm + 3 * (o0 + i);
        const double* bc = S.bc + 8 * ((code >> 8) & 0xff);
        switch (code & 0xff) {
            case WM_OP_SLIP: op_slip(q, nrm, S.gm1, S.Rg); break;
            case WM_OP_NOSLIP: op_noslip(q, bc, S.gm1, S.Rg); break;
            case WM_OP_FARFIELD: op_farfield(q, nrm, (code >> 16) & 1, bc, S.gamma, S.gm1, S.Rg); break;
            default: break;
        }
    }
    const int db = S.block0 + S.dst[2 * le], dc = S.dst[2 * le + 1];
    if (G.stash != nullptr) {
        // two-phase mode: values first, scatter after every source has been read
#pragma unroll
        for (int v = 0; v < 5; ++v) G.stash[(long long)v * G.total + e] = q[v];
    } else {
        double* d = G.q[db];
        const long long n = G.ncell[db];
#pragma unroll
        for (int v = 0; v < 5; ++v) d[v * n + dc] = q[v];
    }
}

__global__ void ghost_gather_kernel(const __grid_constant__ GhostArgs G) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < G.total) ghost_entry(G, e);
}

__global__ void ghost_scatter_kernel(const __grid_constant__ GhostArgs G) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.total) return;
    const GhostSeg& S = G.segs[find_seg(G, e)];
    const int le = e - S.start;
    const int db = S.block0 + S.dst[2 * le], dc = S.dst[2 * le + 1];
    double* d = G.q[db];
    const long long n = G.ncell[db];
#pragma unroll
    for (int v = 0; v < 5; ++v) d[v * n + dc] = G.stash[(long long)v * G.total + e];
}

cudaError_t launch_ghost(const GhostArgs& G, cudaStream_t s) {
    if (G.total == 0) return cudaSuccess;
    const int nt = 256, nb = (G.total + nt - 1) / nt;
    ghost_gather_kernel<<<nb, nt, 0, s>>>(G);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || G.stash == nullptr) return e;
    ghost_scatter_kernel<<<nb, nt, 0, s>>>(G);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ wall model
// WallModel.wall_flux (wmles/bc.py:145-166) with EquilibriumWallModel (wmles/wall_model.py:42-61)
__device__ __forceinline__ void wall_face(const WallArgs& A, int w, long long f) {
    const WallDev& W = A.walls[w];
    const long long nf = (long long)W.nt1 * W.nt2;
    if (f >= nf) return;
    const BlockDev& B = A.blocks[W.block];
    const CaseDev& C = A.cases[B.case_id];
    const int ng = B.ng, n = B.n[W.axis];
    const int a = int(f / W.nt2) + ng, b = int(f % W.nt2) + ng;
    const int mi = W.side == 0 ? ng + W.n_match - 1 : ng + n - W.n_match;
    const int ci = W.side == 0 ? ng : ng + n - 1;
    const double* q = A.q[W.block];
    const long long N = B.ncell;
    const long long im = cell_index(B, W.axis, mi, a, b), ic = cell_index(B, W.axis, ci, a, b);
    const double rho = q[im];
    const double u[3] = {q[N + im] / rho, q[2 * N + im] / rho, q[3 * N + im] / rho};
    const double ke = (u[0] * u[0] + u[1] * u[1]) + u[2] * u[2];
    const double p_h = C.gm1 * (q[4 * N + im] - 0.5 * rho * ke);
    const double T_h = p_h / (rho * C.Rg);
    const double rb = q[ic];
    const double ub[3] = {q[N + ic] / rb, q[2 * N + ic] / rb, q[3 * N + ic] / rb};
    const double p_b = C.gm1 * (q[4 * N + ic] - 0.5 * rb * ((ub[0] * ub[0] + ub[1] * ub[1]) + ub[2] * ub[2]));
    const double Sm = W.geom[f], nrm[3] = {W.geom[nf + f], W.geom[2 * nf + f], W.geom[3 * nf + f]};
    const double h = W.geom[4 * nf + f];
    const double un = (u[0] * nrm[0] + u[1] * nrm[1]) + u[2] * nrm[2];
    const double up[3] = {u[0] - un * nrm[0], u[1] - un * nrm[1], u[2] - un * nrm[2]};
    const double U = sqrt((up[0] * up[0] + up[1] * up[1]) + up[2] * up[2] + 1e-20);
    // equilibrium model
    const double Um = fmax(U, 1e-8);
    const double T_w = W.isothermal ? W.T_wall : T_h + C.Pr13 * (Um * Um) / (2.0 * C.cp);
    const double rho_w = p_h / (C.Rg * T_w);
    const double mu_w = sutherland_d(T_w, C);
    bool moving;
    const double ut = spalding_utau(W.kappa, W.ekb, W.n_iter, h, Um, rho_w, mu_w, &moving);
    if (moving) atomicOr(C.status, WM_ST_WALL);
    const double tau = rho_w * (ut * ut);
    double qw = 0.0;
    if (W.isothermal) {
        // Kader (1981) temperature law
        const double Pr = C.Pr;
        const double yp = fmax(h * ut * rho_w / mu_w, 1e-6);
        const double x = Pr * yp, x2 = x * x;
        const double Gam = fmax(0.01 * (x2 * x2) / (1.0 + 5.0 * C.Pr3 * yp), 1e-20);
        const double Tp = Pr * yp * exp(-Gam) + (2.12 * log(1.0 + yp) + C.kader_beta) * exp(-1.0 / Gam);
        qw = rho_w * C.cp * ut * (T_w - T_h) / Tp;
    }
    const double sgn = W.side == 1 ? 1.0 : -1.0;
    W.F[f] = 0.0;
#pragma unroll
    for (int v = 0; v < 3; ++v) W.F[(1 + v) * nf + f] = sgn * ((p_b * nrm[v] + tau * (up[v] / U)) * Sm);
    W.F[4 * nf + f] = sgn * (-qw * Sm);
    W.tq[f] = tau;
    W.tq[nf + f] = qw;
}

__global__ void wall_kernel(const __grid_constant__ WallArgs A) {
    wall_face(A, blockIdx.y, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

cudaError_t launch_wall(const WallArgs& W, cudaStream_t s) {
    if (W.nwalls == 0) return cudaSuccess;
    dim3 grid((W.max_faces + 127) / 128, W.nwalls);
    wall_kernel<<<grid, 128, 0, s>>>(W);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ sponge
// volume-weighted spanwise mean of q over interior k, per interior (i, j) row
// (SmoothRampSponge.__call__, wmles/smooth_ramp.py:212-216), for the rows listed at case
// creation (sponge_flags_kernel); one warp per row (the shuffles below see all 32 lanes)
__device__ __forceinline__ void sponge_row(const SpongeArgs& S, int b, int row, int lane) {
    const BlockDev& B = S.blocks[b];
    const int ng = B.ng, nj = B.n[1], nk = B.n[2];
    const int i = row / nj + ng, j = row % nj + ng;
    const long long N = B.ncell;
    const long long base = i * B.plane + (long long)j * B.N[2];
    const double* q = S.q[b];
    double acc[5] = {0, 0, 0, 0, 0}, vs = 0.0;
    for (int k = ng + lane; k < ng + nk; k += 32) {
        const double vol = B.met[WM_MET_VOL * N + base + k];
        vs += vol;
#pragma unroll
        for (int v = 0; v < 5; ++v) acc[v] += q[v * N + base + k] * vol;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        vs += __shfl_down_sync(0xffffffffu, vs, o);
#pragma unroll
        for (int v = 0; v < 5; ++v) acc[v] += __shfl_down_sync(0xffffffffu, acc[v], o);
    }
    if (lane == 0) {
        const long long mn = (long long)B.N[0] * B.N[1];
        const long long mi = (long long)i * B.N[1] + j;
#pragma unroll
        for (int v = 0; v < 5; ++v) S.mean[b][v * mn + mi] = acc[v] / vs;
    }
}

// A row whose every cell lies before the sponge start needs no mean: the stage kernel's
// sponge term there is sigma * (q - mean) with sigma exactly 0 (the same expression as its
// ramp argument decides it), and the row's mean stays at its initial 0.  The mesh is fixed,
// so the rows that do need one are found once, at case creation: one warp per row.
__global__ void sponge_flags_kernel(const double* xcx, long long plane, int Nk, int ng, int ni, int nj, int nk,
                                    double invL, double xs, double inv_dx, unsigned char* flags) {
    const int row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (row >= ni * nj) return;          // uniform over the warp
    const int i = row / nj + ng, j = row % nj + ng;
    const long long base = i * plane + (long long)j * Nk;
    bool active = false;
    for (int k = ng + lane; k < ng + nk; k += 32) active |= (xcx[base + k] * invL - xs) * inv_dx > 0.0;
    active = __any_sync(0xffffffffu, active);
    if (lane == 0) flags[row] = active ? 1 : 0;
}

cudaError_t launch_sponge_flags(const double* xcx, long long plane, int Nk, int ng, int ni, int nj, int nk,
                                double invL, double xs, double inv_dx, unsigned char* flags, cudaStream_t s) {
    const int rows = ni * nj;
    if (rows == 0) return cudaSuccess;
    sponge_flags_kernel<<<(rows + 3) / 4, 128, 0, s>>>(xcx, plane, Nk, ng, ni, nj, nk, invL, xs, inv_dx, flags);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ fused surface launch
constexpr int SURF_NT = 256;

// CTA order: wall faces first (the longest dependency chains: Newton iterations), then
// sponge rows, then ghost entries, so the slow parts start in the first wave.  Four CTAs per
// SM (64 registers, a few spills in the wall part) rather than three at 80: the ghost entries
// are chains of dependent loads and gain from the extra warps (channel surface time -7 %).
__global__ void __launch_bounds__(SURF_NT, 4) surface_kernel(const __grid_constant__ SurfaceArgs A) {
    int bx = blockIdx.x;
    if (bx < A.w_ctas) {
        const int w = bx / A.w_per;
        wall_face(A.W, w, (long long)(bx - w * A.w_per) * SURF_NT + threadIdx.x);
        return;
    }
    bx -= A.w_ctas;
    if (bx < A.s_ctas) {
        const int it = bx * (SURF_NT / 32) + (threadIdx.x >> 5);     // uniform over the warp
        if (it < A.S.nrows) sponge_row(A.S, A.S.rows[2 * it], A.S.rows[2 * it + 1], threadIdx.x & 31);
        return;
    }
    bx -= A.s_ctas;
    const int e = bx * SURF_NT + threadIdx.x;
    if (e < A.G.total) ghost_entry(A.G, e);
}

cudaError_t launch_surface(SurfaceArgs& A, cudaStream_t s) {
    A.g_ctas = (A.G.total + SURF_NT - 1) / SURF_NT;
    A.w_per = A.W.nwalls ? (A.W.max_faces + SURF_NT - 1) / SURF_NT : 0;
    A.w_ctas = A.w_per * A.W.nwalls;
    A.s_ctas = (A.S.nrows + SURF_NT / 32 - 1) / (SURF_NT / 32);
    const int n = A.g_ctas + A.w_ctas + A.s_ctas;
    if (n == 0) return cudaSuccess;
    surface_kernel<<<n, SURF_NT, 0, s>>>(A);
    return cudaGetLastError();
}

}  // namespace wm
