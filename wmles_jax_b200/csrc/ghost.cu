// Ghost-cell gather: executes a precomputed per-ghost-cell program.
//
// The host traces the reference's ghost-fill order (Solver.apply_bcs, wmles/solver.py:59-73:
// passes x axes x blocks x sides of block-to-block exchange or BC mirror fill) on cell
// indices, so every ghost cell becomes "take one source value (an interior cell of some
// block, a synthetic-inflow value or a constant state) and apply a short chain of per-cell
// maps".  The maps are the reference's BC maps (wmles/bc.py:41-115) evaluated in the same
// FP64 operation order as NumPy; this file is compiled with -fmad=false so no multiply-add
// is contracted, which makes the gather bit-identical to the reference's ghost fill.
#include "wm_internal.cuh"
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

__global__ void ghost_gather_kernel(const __grid_constant__ GhostArgs G) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.total) return;
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

}  // namespace wm
