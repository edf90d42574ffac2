// Block geometry on the device (Mesh.finalize's metrics, wmles/mesh.py:53-73, and the
// packed metric table the stage kernels read), from the node array extended by the ghost
// nodes.  Set-up work: three memory-bound passes over the block, run once per grid.
//
// The arithmetic is the host path's, operation for operation, and this file is compiled
// with -fmad=false, so every output is bit-identical to the NumPy restatement except the
// SGS filter width V^(1/3), which calls the device pow (the host calls the C library's):
//   face pass  S[d] = 0.5 (c11 - c00) x (c01 - c10), xf[d] = 0.25 (((c00 + c10) + c01) + c11)
//              for the four nodes c_ab of each face normal to d (tangents (d+1, d+2) mod 3)
//   cell pass  V = (((((F0+ - F0-) + F1+) - F1-) + F2+) - F2-) / 3 with F = xf.S summed
//              x, y, z in order; xc = (sum of the 8 nodes in (i, j, k) lexicographic
//              order, starting from 0) / 8
//   pack pass  the table of WM_MET_*: lower-face S per direction, V, xc, V^(1/3), 1/V and
//              the viscous correction geometry e = dx / |dx|, 1 / |dx| with
//              dx = xc[c] - xc[c - 1] along d and |dx| = sqrt((dx.x^2 + dx.y^2) + dx.z^2),
//              zero on the first layer (wmles/viscous.py:35-37)
#include "geom.cuh"
#include "wmles_cuda.h"

namespace wm {

namespace {

constexpr int GM_NT = 256;
constexpr int GM_MAX_CTAS = 148 * 8;

unsigned grid_for(long long n) {
    long long g = (n + GM_NT - 1) / GM_NT;
    if (g > GM_MAX_CTAS) g = GM_MAX_CTAS;
    return (unsigned)(g < 1 ? 1 : g);
}

struct Ext {
    long long e[3];
    __device__ long long count() const { return e[0] * e[1] * e[2]; }
    __device__ long long flat(long long i, long long j, long long k) const { return (i * e[1] + j) * e[2] + k; }
};

__device__ Ext face_ext(const GeomArgs& A, int d) {
    Ext E{{A.N[0], A.N[1], A.N[2]}};
    E.e[d] += 1;
    return E;
}

__global__ void __launch_bounds__(GM_NT) face_kernel(const __grid_constant__ GeomArgs A) {
    const int d = blockIdx.y;
    const int t1 = (d + 1) % 3, t2 = (d + 2) % 3;
    const Ext E = face_ext(A, d);
    const long long nf = E.count();
    const long long M1 = A.N[1] + 1, M2 = A.N[2] + 1;
    const long long nodes = (long long)(A.N[0] + 1) * M1 * M2;
    const long long stride[3] = {M1 * M2, M2, 1};
    const long long o1 = stride[t1], o2 = stride[t2];
    double* S = A.S[d];
    double* xf = A.xf[d];
    for (long long f = (long long)blockIdx.x * GM_NT + threadIdx.x; f < nf; f += (long long)gridDim.x * GM_NT) {
        const long long e2 = f % E.e[2], r = f / E.e[2];
        const long long e1 = r % E.e[1], e0 = r / E.e[1];
        const long long c00 = e0 * stride[0] + e1 * stride[1] + e2;
        double a[3], b[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double* Xc = A.X + c * nodes;
            const double x00 = Xc[c00], x10 = Xc[c00 + o1], x01 = Xc[c00 + o2], x11 = Xc[c00 + o1 + o2];
            a[c] = x11 - x00;
            b[c] = x01 - x10;
            xf[c * nf + f] = 0.25 * (((x00 + x10) + x01) + x11);
        }
        S[f] = 0.5 * (a[1] * b[2] - a[2] * b[1]);
        S[nf + f] = 0.5 * (a[2] * b[0] - a[0] * b[2]);
        S[2 * nf + f] = 0.5 * (a[0] * b[1] - a[1] * b[0]);
    }
}

__device__ double face_flux(const GeomArgs& A, int d, long long nf, long long fi) {
    const double* S = A.S[d];
    const double* xf = A.xf[d];
    return (xf[fi] * S[fi] + xf[nf + fi] * S[nf + fi]) + xf[2 * nf + fi] * S[2 * nf + fi];
}

__global__ void __launch_bounds__(GM_NT) cell_kernel(const __grid_constant__ GeomArgs A) {
    const long long N1 = A.N[1], N2 = A.N[2];
    const long long n = (long long)A.N[0] * N1 * N2;
    const long long M1 = N1 + 1, M2 = N2 + 1;
    const long long nodes = (long long)(A.N[0] + 1) * M1 * M2;
    Ext E[3];
    long long nf[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        E[d] = face_ext(A, d);
        nf[d] = E[d].count();
    }
    for (long long c = (long long)blockIdx.x * GM_NT + threadIdx.x; c < n; c += (long long)gridDim.x * GM_NT) {
        const long long k = c % N2, r = c / N2;
        const long long j = r % N1, i = r / N1;
        double v = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const long long lo = E[d].flat(i, j, k);
            const long long hi = E[d].flat(i + (d == 0), j + (d == 1), k + (d == 2));
            const double fh = face_flux(A, d, nf[d], hi), fl = face_flux(A, d, nf[d], lo);
            v = d == 0 ? fh - fl : (v + fh) - fl;
        }
        A.vol[c] = v / 3.0;
        const long long n000 = (i * M1 + j) * M2 + k;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const double* Xq = A.X + q * nodes;
            double acc = 0.0;
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b)
#pragma unroll
                    for (int e = 0; e < 2; ++e) acc = acc + Xq[n000 + (a * M1 + b) * M2 + e];
            A.xc[q * n + c] = acc / 8.0;
        }
    }
}

__global__ void __launch_bounds__(GM_NT) pack_kernel(const __grid_constant__ GeomArgs A) {
    const long long N1 = A.N[1], N2 = A.N[2];
    const long long n = (long long)A.N[0] * N1 * N2;
    const long long cstride[3] = {N1 * N2, N2, 1};
    Ext E[3];
    long long nf[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        E[d] = face_ext(A, d);
        nf[d] = E[d].count();
    }
    double* M = A.met;
    for (long long c = (long long)blockIdx.x * GM_NT + threadIdx.x; c < n; c += (long long)gridDim.x * GM_NT) {
        const long long k = c % N2, r = c / N2;
        const long long j = r % N1, i = r / N1;
        const long long pos[3] = {i, j, k};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const long long fi = E[d].flat(i, j, k);
#pragma unroll
            for (int q = 0; q < 3; ++q) M[(WM_MET_SIX + 3 * d + q) * n + c] = A.S[d][q * nf[d] + fi];
        }
        const double vol = A.vol[c];
        M[WM_MET_VOL * n + c] = vol;
        double x[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            x[q] = A.xc[q * n + c];
            M[(WM_MET_XCX + q) * n + c] = x[q];
        }
        M[WM_MET_DELTA * n + c] = pow(vol, 1.0 / 3.0);
        M[WM_MET_IVOL * n + c] = 1.0 / vol;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int base = WM_MET_EIX + 4 * d;
            if (pos[d] == 0) {
#pragma unroll
                for (int q = 0; q < 4; ++q) M[(base + q) * n + c] = 0.0;
                continue;
            }
            double dx[3];
#pragma unroll
            for (int q = 0; q < 3; ++q) dx[q] = x[q] - A.xc[q * n + c - cstride[d]];
            const double dist = sqrt((dx[0] * dx[0] + dx[1] * dx[1]) + dx[2] * dx[2]);
#pragma unroll
            for (int q = 0; q < 3; ++q) M[(base + q) * n + c] = dx[q] / dist;
            M[(base + 3) * n + c] = 1.0 / dist;
        }
    }
}

__global__ void __launch_bounds__(GM_NT) to_f32_kernel(const double* __restrict__ src, float* __restrict__ dst,
                                                        long long n) {
    for (long long i = (long long)blockIdx.x * GM_NT + threadIdx.x; i < n; i += (long long)gridDim.x * GM_NT)
        dst[i] = __double2float_rn(src[i]);
}

}  // namespace

cudaError_t launch_geometry(const GeomArgs& A, cudaStream_t s) {
    long long maxf = 0;
    for (int d = 0; d < 3; ++d) {
        long long e[3] = {A.N[0], A.N[1], A.N[2]};
        e[d] += 1;
        const long long f = e[0] * e[1] * e[2];
        if (f > maxf) maxf = f;
    }
    const long long n = (long long)A.N[0] * A.N[1] * A.N[2];
    face_kernel<<<dim3(grid_for(maxf), 3), GM_NT, 0, s>>>(A);
    cell_kernel<<<grid_for(n), GM_NT, 0, s>>>(A);
    if (A.met) pack_kernel<<<grid_for(n), GM_NT, 0, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_to_f32(const double* src, float* dst, long long n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    to_f32_kernel<<<grid_for(n), GM_NT, 0, s>>>(src, dst, n);
    return cudaGetLastError();
}

}  // namespace wm
