// Derived output fields on the device (derived_fields, wmles/io_vtk.py:269-293): per interior
// cell rho, velocity, pressure, temperature, Mach number, SGS viscosity mu_t, molecular
// viscosity, vorticity magnitude and Q-criterion, from a state whose first ghost layer is
// filled, so output needs no copy of the state to the host.
//
// One interior cell per thread, FP64.  The velocity gradient is the Green-Gauss gradient of
// wmles/viscous.py:6-19 (face values = means of the two cells, times the face area vector,
// over the volume), the SGS viscosity the case's model (wmles/sgs.py:14-50).
#include "physics.cuh"
#include "aux.cuh"
#include "derived.cuh"

namespace wm {

constexpr int DV_NT = 256;

__global__ void __launch_bounds__(DV_NT) derived_kernel(const __grid_constant__ DerivedArgs A) {
    const BlockDev& B = *A.block;
    const CaseDev& C = *A.cs;
    const int ng = B.ng, nj = B.n[1], nk = B.n[2];
    const long long ni_cells = (long long)B.n[0] * nj * nk;
    const long long c = (long long)blockIdx.x * DV_NT + threadIdx.x;
    if (c >= ni_cells) return;
    const int i = int(c / ((long long)nj * nk)) + ng;
    const int r = int(c % ((long long)nj * nk));
    const int j = r / nk + ng, k = r % nk + ng;
    const long long N = B.ncell, plane = B.plane, Nk = B.N[2];
    const long long idx = i * plane + (long long)j * Nk + k;
    const double* q = A.q;
    const double* met = B.met;
    auto vel = [&](long long x, double u[3]) {
        const double rho = q[x];
        u[0] = q[N + x] / rho;
        u[1] = q[2 * N + x] / rho;
        u[2] = q[3 * N + x] / rho;
    };
    double u0[3], um[3][3], up[3][3];
    vel(idx, u0);
    const long long off[3] = {plane, Nk, 1};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        vel(idx - off[d], um[d]);
        vel(idx + off[d], up[d]);
    }
    // g[a][d] = d u_a / d x_d
    double g[9];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double lo = 0.5 * (um[d][a] + u0[a]), hi = 0.5 * (u0[a] + up[d][a]);
#pragma unroll
            for (int x = 0; x < 3; ++x) {
                const double sl = met[(3 * d + x) * N + idx], sh = met[(3 * d + x) * N + idx + off[d]];
                acc[x] += hi * sh - lo * sl;
            }
        }
        const double vol = met[WM_MET_VOL * N + idx];
#pragma unroll
        for (int x = 0; x < 3; ++x) g[3 * a + x] = acc[x] / vol;
    }
    const double rho = q[idx];
    const double ke = (u0[0] * u0[0] + u0[1] * u0[1]) + u0[2] * u0[2];
    const double p = C.gm1 * (q[4 * N + idx] - (0.5 * rho) * ke);
    const double T = p / (rho * C.Rg);
    const double mu = sutherland_d(T, C);
    const double mut = A.sgs != WM_SGS_NONE ? rho * sgs_nut<double>(A.sgs, g, met[WM_MET_DELTA * N + idx], C.sgs_c) : 0.0;
    const double wxy = g[3] - g[1], wxz = g[6] - g[2], wyz = g[7] - g[5];
    const double om = sqrt((wxy * wxy + wxz * wxz) + wyz * wyz);
    double s2 = 0.0, o2 = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const double s = 0.5 * (g[3 * a + b] + g[3 * b + a]), o = 0.5 * (g[3 * a + b] - g[3 * b + a]);
            s2 += s * s;
            o2 += o * o;
        }
    const double qc = 0.5 * (o2 - s2);
    const double mach = sqrt(ke) / sqrt(C.gamma * C.Rg * T);
    const double out[WM_NDERIVED] = {rho, u0[0], u0[1], u0[2], p, T, mach, mut, mu, om, qc};
    const long long oi = ((long long)(i - ng) * nj + (j - ng)) * nk + (k - ng);
#pragma unroll
    for (int v = 0; v < WM_NDERIVED; ++v) A.out[v * ni_cells + oi] = out[v];
}

cudaError_t launch_derived(const DerivedArgs& A, long long cells, cudaStream_t s) {
    if (cells == 0) return cudaSuccess;
    derived_kernel<<<(unsigned)((cells + DV_NT - 1) / DV_NT), DV_NT, 0, s>>>(A);
    return cudaGetLastError();
}

}  // namespace wm
