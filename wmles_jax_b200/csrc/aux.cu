// Surface and reduction kernels of the step: wall-model flux override, CFL time step with
// the constant-mass-flux update, sponge spanwise means and synthetic-turbulence inflow.
#include <algorithm>
#include <cfloat>
#include "physics.cuh"
#include "aux.cuh"

namespace wm {

// ------------------------------------------------------------------ reductions
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < NT / 32; ++w) s += red[w];
    __syncthreads();
    if (threadIdx.x == 0) red[0] = s;
    __syncthreads();
    const double r = red[0];
    __syncthreads();
    return r;
}

template <typename M> __device__ __forceinline__ const M* metrics_of(const BlockDev& B);
template <> __device__ __forceinline__ const double* metrics_of<double>(const BlockDev& B) { return B.met; }
template <> __device__ __forceinline__ const float* metrics_of<float>(const BlockDev& B) { return B.met32; }

// min that propagates NaN like NumPy's np.min (a NaN time step must not be masked)
__device__ __forceinline__ double nanmin(double a, double b) { return (a != a || a < b) ? a : b; }

// order-preserving 64-bit key of a double for an integer atomicMin: NaN gets the lowest key,
// so a NaN time step wins the minimum as it does in NumPy's np.min
__device__ __forceinline__ unsigned long long dt_key_of(double x) {
    if (x != x) return 0ull;
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dt_value_of(unsigned long long k) {
    if (k == 0ull) return __longlong_as_double(0x7ff8000000000000ll);
    return __longlong_as_double((long long)((k >> 63) ? (k & 0x7fffffffffffffffull) : ~k));
}

// CFL time step (Solver._dt, wmles/solver.py:135-151), optionally after applying the
// constant-mass-flux shift (ConstantMassFlux.__call__, wmles/solver.py:22-36) in place.
// The view's interior cells are cut into chunks of DT_NT cells, one cell per thread, chunks
// numbered block by block (so case by case); one wave of resident CTAs walks the chunks
// (grid stride).  Each thread keeps the minimum of its cells while the chunks stay in one
// case; when the case changes and at the end, each warp folds its threads' minima and makes
// one atomicMin on the case's key.  The last CTA to finish turns the keys into time steps
// and resets them.  A minimum is exact in any order, so the result does not depend on the
// grid, the chunking or the batch.  M: the metric copy read (double; float for the mixed
// form); the arithmetic is FP64 either way.
template <typename M>
__global__ void __launch_bounds__(DT_NT) dt_kernel(const __grid_constant__ DtArgs D) {
    __shared__ bool last;
    double run = DBL_MAX;          // this thread's minimum over its cells of case `cur`
    int cur = -1;
    auto flush = [&]() {
        double m = run;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = nanmin(m, __shfl_down_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0) {
            atomicMin(D.dt_key + cur, dt_key_of(m));
            __threadfence();
        }
        run = DBL_MAX;
    };
#pragma unroll 1
    for (int chunk = blockIdx.x; chunk < D.ncta; chunk += gridDim.x) {
        int b = 0;
        {
            int hi = D.nblocks - 1;
            while (b < hi) {             // last block whose first chunk is <= chunk
                const int mid = (b + hi + 1) >> 1;
                if (D.cta_start[mid] <= chunk) b = mid; else hi = mid - 1;
            }
        }
        const BlockDev& B = D.blocks[b];
        if (D.want_dt && B.case_id != cur) {    // uniform over the CTA: one chunk at a time
            if (cur >= 0) flush();
            cur = B.case_id;
        }
        const CaseDev& C = D.cases[B.case_id];
        const bool cmf = D.cmf_delta != nullptr && C.cmf_dir >= 0;
        const int ng = B.ng, nj = B.n[1], nk = B.n[2];
        const int Nk = B.N[2];
        const long long N = B.ncell, plane = B.plane;
        const long long ncells = (long long)B.n[0] * nj * nk;
        const long long c = (long long)(chunk - D.cta_start[b]) * DT_NT + threadIdx.x;
        if (c < ncells) {
            double* q = D.q[b];
            const M* met = metrics_of<M>(B);
            const int i = int(c / ((long long)nj * nk)) + ng;
            const int r = int(c % ((long long)nj * nk));
            const int j = r / nk + ng, k = r % nk + ng;
            const long long idx = i * plane + (long long)j * Nk + k;
            double qv[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) qv[v] = q[v * N + idx];
            // every metric this cell needs, read-only and issued before any store to q
            const long long off[3] = {plane, Nk, 1};
            double Sl[9], Sh[9];
#pragma unroll
            for (int d = 0; d < 3; ++d)
#pragma unroll
                for (int x = 0; x < 3; ++x) {
                    Sl[3 * d + x] = __ldg(met + (3 * d + x) * N + idx);
                    Sh[3 * d + x] = __ldg(met + (3 * d + x) * N + idx + off[d]);
                }
            const double vol = __ldg(met + WM_MET_VOL * N + idx);
            if (cmf) {
                const double delta = D.cmf_delta[B.case_id];
                const int m = 1 + C.cmf_dir;
                const double dE = (2.0 * qv[m] * delta + delta * delta) / (2.0 * qv[0]);
                qv[m] = qv[m] + delta;
                qv[4] = qv[4] + dE;
                q[m * N + idx] = qv[m];
                q[4 * N + idx] = qv[4];
            }
            const double rho = qv[0];
            const double ir = 1.0 / rho;
            const double u = qv[1] * ir, v = qv[2] * ir, w = qv[3] * ir;
            const double p = C.gm1 * (qv[4] - 0.5 * rho * ((u * u + v * v) + w * w));
            {
                // the state must still be a flow state (bits kept in the case's status word)
                unsigned bad = 0u;
#pragma unroll
                for (int x = 0; x < 5; ++x)
                    if (!isfinite(qv[x])) bad = WM_ST_NONFINITE;
                if (!(rho > 0.0)) bad |= WM_ST_RHO;
                if (!(p > 0.0)) bad |= WM_ST_PRESSURE;
                if (bad) atomicOr(C.status, bad);
            }
            if (D.want_dt) {
                const double ivol = 1.0 / vol;
                const double T = p * ir * C.inv_Rg;
                const double cs = sqrt(C.gamma * C.Rg * T);
                const double nu = C.nu_fac * sutherland_d(T, C) * ir;
                double lam = 0.0, lamv = 0.0;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double sx = 0.5 * (Sl[3 * d] + Sh[3 * d]);
                    const double sy = 0.5 * (Sl[3 * d + 1] + Sh[3 * d + 1]);
                    const double sz = 0.5 * (Sl[3 * d + 2] + Sh[3 * d + 2]);
                    const double Sm = sqrt((sx * sx + sy * sy) + sz * sz);
                    lam = lam + fabs((u * sx + v * sy) + w * sz) + cs * Sm;
                    lamv = lamv + nu * (Sm * Sm) * ivol;
                }
                run = nanmin(run, C.cfl * vol / (lam + 4.0 * lamv));
            }
        }
    }
#pragma unroll 1
    for (int chunk = blockIdx.x; chunk < D.ngcta; chunk += gridDim.x) {
        int b = 0;
        {
            int hi = D.nblocks - 1;
            while (b < hi) {
                const int mid = (b + hi + 1) >> 1;
                if (D.gcta_start[mid] <= chunk) b = mid; else hi = mid - 1;
            }
        }
        const BlockDev& B = D.blocks[b];
        const long long g = (long long)(chunk - D.gcta_start[b]) * DT_NT + threadIdx.x;
        if (g < ghost_cells(B)) {
            const CaseDev& C = D.cases[B.case_id];
            const long long N = B.ncell, idx = ghost_cell_index(B, g);
            const double* src = D.q_src[b];
            double* q = D.q[b];
            double qv[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) qv[v] = src[v * N + idx];
            if (D.cmf_delta != nullptr && C.cmf_dir >= 0) {
                // the reference shifts every cell, ghost cells included (wmles/solver.py:30-36)
                const double delta = D.cmf_delta[B.case_id];
                const int m = 1 + C.cmf_dir;
                const double dE = (2.0 * qv[m] * delta + delta * delta) / (2.0 * qv[0]);
                qv[m] = qv[m] + delta;
                qv[4] = qv[4] + dE;
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) q[v * N + idx] = qv[v];
        }
    }
    if (!D.want_dt) return;
    if (cur >= 0) flush();
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(D.counter, 1u);
        last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        for (int c = threadIdx.x; c < D.ncases; c += DT_NT) {
            volatile unsigned long long* kp = D.dt_key + c;
            const unsigned long long key = *kp;
            const double dt = dt_value_of(key);
            if (D.dt_out[c] != nullptr) D.dt_out[c][0] = dt;
            if (!(dt > 0.0 && dt <= DBL_MAX)) atomicOr(D.cases[c].status, WM_ST_DT);
            *kp = DT_KEY_EMPTY;
        }
        if (threadIdx.x == 0) *D.counter = 0u;
    }
}

// status words of a batch's member cases into one array (wm_batch_status)
__global__ void status_gather_kernel(const CaseDev* cases, int ncases, unsigned* out) {
    for (int c = threadIdx.x; c < ncases; c += blockDim.x) out[c] = *(volatile unsigned*)cases[c].status;
}

cudaError_t launch_status_gather(const CaseDev* cases, int ncases, unsigned* out, cudaStream_t s) {
    status_gather_kernel<<<1, 128, 0, s>>>(cases, ncases, out);
    return cudaGetLastError();
}

// resident CTAs of one wave of dt_kernel<M> (computed once per process and metric type)
template <typename M>
static int dt_wave() {
    static int ctas = 0;
    if (ctas == 0) {
        int dev = 0, sms = 148, per_sm = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dt_kernel<M>, DT_NT, 0);
        ctas = sms * (per_sm > 0 ? per_sm : 1);
    }
    return ctas;
}

cudaError_t launch_dt(const DtArgs& D, cudaStream_t s) {
    if (D.met32)
        dt_kernel<float><<<std::max(1, std::min(std::max(D.ncta, D.ngcta), dt_wave<float>())), DT_NT, 0, s>>>(D);
    else
        dt_kernel<double><<<std::max(1, std::min(std::max(D.ncta, D.ngcta), dt_wave<double>())), DT_NT, 0, s>>>(D);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ synthetic inflow
// SmoothRampInflow.fill_at_time / _unit_noise (wmles/smooth_ramp.py:150-197), in two
// launches: the mode sums (n_modes cosines per component and ghost cell) cut into IN_PARTS
// contiguous mode ranges, one thread per (range, row, component, k), so that no thread
// evaluates more than n_modes / IN_PARTS cosines; then one CTA per (ghost layer, j) row adds
// the ranges in order, normalises the row and writes the ghost states.
constexpr int IN_NT = 256;

__global__ void __launch_bounds__(IN_NT) inflow_modes_kernel(const __grid_constant__ InflowArgs I, long long units) {
    const long long u = (long long)blockIdx.x * IN_NT + threadIdx.x;
    if (u >= units) return;
    const BlockDev& B = *I.block;
    const int ng = B.ng, Nj = B.N[1], Nk = B.N[2];
    const long long rows = (long long)ng * Nj;
    // u = ((part * rows + row) * 3 + c) * Nk + k, row = m * Nj + j
    const int k = int(u % Nk);
    const long long r1 = u / Nk;
    const int c = int(r1 % 3);
    const long long r2 = r1 / 3;
    const int row = int(r2 % rows), pt = int(r2 / rows);
    const int m = row / Nj, j = row - m * Nj, gi = ng - 1 - m;
    const long long N = B.ncell;
    const double time = I.time0 + I.time_dt * (I.dt ? *I.dt : 0.0);
    const double X = I.U_inf * time / I.L;
    const double* kx = I.modes + (c * 4 + 0) * I.n_modes;
    const double* ky = I.modes + (c * 4 + 1) * I.n_modes;
    const double* kz = I.modes + (c * 4 + 2) * I.n_modes;
    const double* ph = I.modes + (c * 4 + 3) * I.n_modes;
    const long long idx = ((long long)gi * Nj + j) * Nk + k;
    const double y = B.met[WM_MET_XCY * N + idx] / I.L, z = B.met[WM_MET_XCZ * N + idx] / I.L;
    const int per = (I.n_modes + IN_PARTS - 1) / IN_PARTS;
    const int q1 = min(I.n_modes, (pt + 1) * per);
    double acc = 0.0;
    for (int q = pt * per; q < q1; ++q) acc += cos(((kx[q] * X + ky[q] * y) + kz[q] * z) + ph[q]);
    I.raw[u] = acc;
}

// np.interp on the profile table (column 0 the abscissa, end values clamped): the bracket
// of y is searched once per cell and shared by every column
struct InterpAt {
    int lo, hi;      // hi < 0: clamped to row lo
    __device__ InterpAt(const double* tab, int n, double y) {
        if (y <= tab[0]) { lo = 0; hi = -1; return; }
        if (y >= tab[7 * (n - 1)]) { lo = n - 1; hi = -1; return; }
        lo = 0; hi = n - 1;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (tab[7 * mid] <= y) lo = mid; else hi = mid;
        }
    }
    __device__ double col(const double* tab, double y, int c) const {
        if (hi < 0) return tab[7 * lo + c];
        const double x0 = tab[7 * lo], x1 = tab[7 * hi];
        const double f0 = tab[7 * lo + c], f1 = tab[7 * hi + c];
        const double slope = (f1 - f0) / (x1 - x0);
        return slope * (y - x0) + f0;
    }
};

__global__ void __launch_bounds__(IN_NT) inflow_kernel(const __grid_constant__ InflowArgs I) {
    extern __shared__ double fsm[];            // 3 x Nk
    __shared__ double red[IN_NT / 32];
    const BlockDev& B = *I.block;
    const int ng = B.ng, Nj = B.N[1], Nk = B.N[2], nk = B.n[2];
    const int j = blockIdx.x, m = blockIdx.y, gi = ng - 1 - m;
    const long long N = B.ncell;
    double* f0 = fsm;
    // raw mode sums of the row's three components: the partial sums added in range order
    const long long rows = (long long)ng * Nj, row = (long long)m * Nj + j;
    for (int it = threadIdx.x; it < 3 * Nk; it += IN_NT) {
        double acc = I.raw[row * 3 * Nk + it];
        for (int pt = 1; pt < IN_PARTS; ++pt) acc += I.raw[(pt * rows + row) * 3 * Nk + it];
        fsm[it] = acc;
    }
    __syncthreads();
    for (int c = 0; c < 3; ++c) {
        double* f = fsm + c * Nk;
        double s_int = 0.0;
        for (int k = threadIdx.x; k < Nk; k += IN_NT)
            if (k >= ng && k < ng + nk) s_int += f[k];
        const double mean = block_sum<IN_NT>(s_int, red) / nk;
        double cov_acc = 0.0;
        for (int k = threadIdx.x; k < Nk; k += IN_NT) {
            f[k] -= mean;
            if (c == 1 && k >= ng && k < ng + nk) cov_acc += f[k] * f0[k];
        }
        if (c == 1) {
            const double cov = block_sum<IN_NT>(cov_acc, red) / nk;
            for (int k = threadIdx.x; k < Nk; k += IN_NT) f[k] -= cov * f0[k];
        }
        double v_acc = 0.0;
        for (int k = threadIdx.x; k < Nk; k += IN_NT)
            if (k >= ng && k < ng + nk) v_acc += f[k] * f[k];
        const double var = block_sum<IN_NT>(v_acc, red) / nk;
        const double inv = 1.0 / sqrt(fmax(var, 1e-20));
        for (int k = threadIdx.x; k < Nk; k += IN_NT) f[k] *= inv;
        __syncthreads();
    }
    const long long on = (long long)ng * Nj * Nk;
    const double U = I.U_inf;
    for (int k = threadIdx.x; k < Nk; k += IN_NT) {
        const long long idx = ((long long)gi * Nj + j) * Nk + k;
        const double y = B.met[WM_MET_XCY * N + idx] / I.L;
        const InterpAt at(I.table, I.n_tab, y);
        const double uu = fmax(at.col(I.table, y, 3), 0.0) * (U * U);
        const double vv = fmax(at.col(I.table, y, 4), 0.0) * (U * U);
        const double ww = fmax(at.col(I.table, y, 5), 0.0) * (U * U);
        const double uv = at.col(I.table, y, 6) * (U * U);
        const double su = sqrt(uu);
        const double l10 = su > 1e-14 ? uv / fmax(su, 1e-14) : 0.0;
        const double l11 = sqrt(fmax(vv - l10 * l10, 0.0));
        const double n0 = fsm[k], n1 = fsm[Nk + k], n2 = fsm[2 * Nk + k];
        const double u = U * at.col(I.table, y, 1) + su * n0;
        const double v = U * at.col(I.table, y, 2) + l10 * n0 + l11 * n1;
        const double w = sqrt(ww) * n2;
        const double rho = I.rho_inf, p = I.p_inf;
        I.out[idx] = rho;
        I.out[on + idx] = rho * u;
        I.out[2 * on + idx] = rho * v;
        I.out[3 * on + idx] = rho * w;
        I.out[4 * on + idx] = p / I.gm1 + 0.5 * rho * ((u * u + v * v) + w * w);
    }
}

cudaError_t launch_inflow(const InflowArgs& I, int Nj, int Nk, int ng, cudaStream_t s) {
    const long long units = (long long)IN_PARTS * ng * Nj * 3 * Nk;
    inflow_modes_kernel<<<(unsigned)((units + IN_NT - 1) / IN_NT), IN_NT, 0, s>>>(I, units);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dim3 grid(Nj, ng);
    const size_t sm = sizeof(double) * 3 * Nk;
    inflow_kernel<<<grid, IN_NT, sm, s>>>(I);
    return cudaGetLastError();
}

}  // namespace wm
