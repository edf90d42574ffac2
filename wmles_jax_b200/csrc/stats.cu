// Plane statistics of a channel block (PlaneStats.accumulate, wmles/channel5200.py:121-152):
// per interior j-plane, the means over interior (i, k) of rho, u, v, w, uu, vv, ww, uv, uw,
// vw, T, p, added to a device accumulator, so a driver samples the flow every few steps
// without copying the state to the host.
//
// One CTA per (i-chunk, plane): each thread walks its cells of the chunk and keeps the 12
// FP64 sums in registers; a block reduction writes one partial per quantity; the last CTA of
// the launch adds, per plane and quantity, the chunk partials in chunk order divided by the
// plane's cell count (a fixed order: the result does not depend on scheduling).
#include <cfloat>
#include "wm_internal.cuh"
#include "stats.cuh"

namespace wm {

constexpr int PS_NT = 256;

__global__ void __launch_bounds__(PS_NT) plane_stats_kernel(const __grid_constant__ PlaneStatsArgs A) {
    __shared__ double red[PS_NQ][PS_NT / 32];
    __shared__ bool last;
    const BlockDev& B = *A.block;
    const int ng = B.ng, ni = B.n[0], nk = B.n[2], Nj = B.N[1], Nk = B.N[2];
    const int chunk = blockIdx.x, jj = blockIdx.y;          // jj: interior plane index
    const int i0 = (int)((long long)chunk * ni / A.nchunks), i1 = (int)((long long)(chunk + 1) * ni / A.nchunks);
    const long long N = B.ncell;
    double acc[PS_NQ];
#pragma unroll
    for (int q = 0; q < PS_NQ; ++q) acc[q] = 0.0;
    const int cells = (i1 - i0) * nk;
    for (int c = threadIdx.x; c < cells; c += PS_NT) {
        const int i = i0 + c / nk + ng, k = c % nk + ng;
        const long long idx = ((long long)i * Nj + (jj + ng)) * Nk + k;
        // gas.cons_to_prim (wmles/gas.py:28-33)
        const double rho = A.q[idx];
        const double u = A.q[N + idx] / rho, v = A.q[2 * N + idx] / rho, w = A.q[3 * N + idx] / rho;
        const double p = A.gm1 * (A.q[4 * N + idx] - (0.5 * rho) * ((u * u + v * v) + w * w));
        const double T = p / (rho * A.Rg);
        const double x[PS_NQ] = {rho, u, v, w, u * u, v * v, w * w, u * v, u * w, v * w, T, p};
#pragma unroll
        for (int q = 0; q < PS_NQ; ++q) acc[q] += x[q];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < PS_NQ; ++q) {
        double s = acc[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) red[q][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x < PS_NQ) {
        double s = 0.0;
        for (int wv = 0; wv < PS_NT / 32; ++wv) s += red[threadIdx.x][wv];
        A.part[((long long)threadIdx.x * B.n[1] + jj) * A.nchunks + chunk] = s;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(A.counter, 1u) == gridDim.x * gridDim.y - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const volatile double* part = A.part;
    const double inv = 1.0 / ((double)ni * nk);
    for (int e = threadIdx.x; e < PS_NQ * B.n[1]; e += PS_NT) {
        double s = 0.0;
        for (int ch = 0; ch < A.nchunks; ++ch) s += part[(long long)e * A.nchunks + ch];
        A.sum[e] += s * inv;
    }
    if (threadIdx.x == 0) *A.counter = 0u;
}

cudaError_t launch_plane_stats(const PlaneStatsArgs& A, int nj, cudaStream_t s) {
    dim3 grid(A.nchunks, nj);
    plane_stats_kernel<<<grid, PS_NT, 0, s>>>(A);
    return cudaGetLastError();
}

}  // namespace wm
