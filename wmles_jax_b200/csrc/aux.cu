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
            M Sl[9], Sh[9];
#pragma unroll
            for (int d = 0; d < 3; ++d)
#pragma unroll
                for (int x = 0; x < 3; ++x) {
                    Sl[3 * d + x] = __ldg(met + (3 * d + x) * N + idx);
                    Sh[3 * d + x] = __ldg(met + (3 * d + x) * N + idx + off[d]);
                }
            const M vol = __ldg(met + WM_MET_VOL * N + idx);
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
                // the cell's CFL rate in the metric precision: FP64 in the FP64 form; FP32 in the
                // mixed form, from its FP32 metric copy like its fluxes (the state, its checks,
                // the constraint and the minimum over cells stay FP64)
                using CF = M;
                const CF ivol = CF(1) / vol;
                const CF irc = CF(ir);
                const CF T = CF(p) * irc * CF(C.inv_Rg);
                const CF cs = sqrt(CF(C.gamma) * CF(C.Rg) * T);
                const CF x = T * CF(C.inv_Tref);
                const CF nu = CF(C.nu_fac) * (CF(C.mu_ref) * (x * sqrt(x)) * CF(C.TrefS) / (T + CF(C.S_suth))) * irc;
                const CF uc = CF(u), vc = CF(v), wc = CF(w);
                CF lam = CF(0), lamv = CF(0);
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const CF sx = CF(0.5) * (Sl[3 * d] + Sh[3 * d]);
                    const CF sy = CF(0.5) * (Sl[3 * d + 1] + Sh[3 * d + 1]);
                    const CF sz = CF(0.5) * (Sl[3 * d + 2] + Sh[3 * d + 2]);
                    const CF Sm = sqrt((sx * sx + sy * sy) + sz * sz);
                    lam = lam + fabs((uc * sx + vc * sy) + wc * sz) + cs * Sm;
                    lamv = lamv + nu * (Sm * Sm) * ivol;
                }
                run = nanmin(run, double(CF(C.cfl) * vol / (lam + CF(4) * lamv)));
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
// launches.  The mode sums: on a general inflow plane n_modes cosines per component and ghost
// cell, cut into IN_PARTS contiguous mode ranges, one thread per (range, row, component, k), so
// that no thread evaluates more than n_modes / IN_PARTS cosines (inflow_modes_kernel); on an
// extruded plane factored sums, one sincos per (component, mode, row)
// (inflow_ext_sums_kernel).  Then one CTA per (ghost layer, j) row adds the ranges in order,
// normalises the row and writes the ghost states (inflow_row_kernel).
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

// time-independent factors of the inflow state per ghost cell (np.interp of the profile table
// at the cell's y, wmles/smooth_ramp.py:160-169), computed once at case creation:
// sqrt(uu), l10, l11, sqrt(ww), U * U_mean, U * V_mean
__global__ void inflow_prof_kernel(const __grid_constant__ InflowArgs I, double* prof, long long n) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;   // ghost-slab cell
    if (idx >= n) return;
    const BlockDev& B = *I.block;
    const double y = B.met[WM_MET_XCY * B.ncell + idx] / I.L;
    const InterpAt at(I.table, I.n_tab, y);
    const double U = I.U_inf;
    const double uu = fmax(at.col(I.table, y, 3), 0.0) * (U * U);
    const double vv = fmax(at.col(I.table, y, 4), 0.0) * (U * U);
    const double ww = fmax(at.col(I.table, y, 5), 0.0) * (U * U);
    const double uv = at.col(I.table, y, 6) * (U * U);
    const double su = sqrt(uu);
    const double l10 = su > 1e-14 ? uv / fmax(su, 1e-14) : 0.0;
    prof[idx] = su;
    prof[n + idx] = l10;
    prof[2 * n + idx] = sqrt(fmax(vv - l10 * l10, 0.0));
    prof[3 * n + idx] = sqrt(ww);
    prof[4 * n + idx] = U * at.col(I.table, y, 1);
    prof[5 * n + idx] = U * at.col(I.table, y, 2);
}

// ghost state of slab cell idx (slab size on) from its profile factors and the unit noise
// (n0, n1, n2) of its row, wmles/smooth_ramp.py:166-176
__device__ __forceinline__ void inflow_write(const InflowArgs& I, long long idx, long long on, double n0, double n1,
                                             double n2) {
    const double* P = I.prof;
    const double u = P[4 * on + idx] + P[idx] * n0;
    const double v = P[5 * on + idx] + P[on + idx] * n0 + P[2 * on + idx] * n1;
    const double w = P[3 * on + idx] * n2;
    const double rho = I.rho_inf, p = I.p_inf;
    I.out[idx] = rho;
    I.out[on + idx] = rho * u;
    I.out[2 * on + idx] = rho * v;
    I.out[3 * on + idx] = rho * w;
    I.out[4 * on + idx] = p / I.gm1 + 0.5 * rho * ((u * u + v * v) + w * w);
}

// ---- extruded inflow plane (z a function of k alone, y constant along k on every ghost row):
// each mode's argument splits as alpha + beta with alpha = (kx X + ky y) + phase per row and
// beta = kz z per k, so cos(alpha + beta) = cos alpha cos beta - sin alpha sin beta with the
// beta factors tabulated once (inflow_cz_kernel): a fill takes one sincos per (component,
// mode, row) instead of one cosine per (component, mode, cell).  The argument is rounded as
// two parts instead of the reference's one sum, a difference of a few units in the last place
// of the argument.
__global__ void inflow_cz_kernel(const __grid_constant__ InflowArgs I, int Nk, double* cz) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nm = I.n_modes;
    if (t >= 3 * nm * Nk) return;
    const int k = t % Nk, cq = t / Nk, c = cq / nm, q = cq - c * nm;
    const BlockDev& B = *I.block;
    const double z = B.met[WM_MET_XCZ * B.ncell + k] / I.L;      // row (0, 0): every row has this z
    double sb, cb;
    sincos(I.modes[(c * 4 + 2) * nm + q] * z, &sb, &cb);
    cz[t] = cb;
    cz[3 * nm * Nk + t] = sb;
}

__device__ __forceinline__ void cp_async8_ca(void* smem, const void* gmem) {
    const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(a), "l"(gmem) : "memory");
}

// sum over the 32 lanes, the same value on every lane
__device__ __forceinline__ double warp_allsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// mode sums of an extruded plane: CTA (g, c) takes component c of the ghost rows
// [g * IN_EXT_ROWS, (g + 1) * IN_EXT_ROWS) (row = layer m * Nj + j, as in inflow_modes_kernel);
// the component's cos / sin (kz z) table is staged in shared memory once, then the rows'
// sincos of alpha, then one thread per (row, k) dot product over the modes from shared memory.
// Output: raw[(row * 3 + c) * Nk + k] (one range).
__global__ void __launch_bounds__(IN_EXT_NT) inflow_ext_sums_kernel(const __grid_constant__ InflowArgs I) {
    extern __shared__ double sm[];    // cos beta, sin beta: 2 x n_modes x Nk; then cos, sin alpha: rows x 2 x n_modes
    const BlockDev& B = *I.block;
    const int ng = B.ng, Nj = B.N[1], Nk = B.N[2];
    const int c = blockIdx.y, nm = I.n_modes;
    const int rows = ng * Nj, r0 = blockIdx.x * IN_EXT_ROWS, nr = min(IN_EXT_ROWS, rows - r0);
    double* tb = sm;
    double* ta = sm + 2 * nm * Nk;
    const double* cz = I.cz + (size_t)c * nm * Nk;
    // the table arrives by cp.async while the sincos below are computed
    for (int t = threadIdx.x; t < nm * Nk; t += IN_EXT_NT) {
        cp_async8_ca(tb + t, cz + t);
        cp_async8_ca(tb + nm * Nk + t, cz + (size_t)3 * nm * Nk + t);
    }
    const double time = I.time0 + I.time_dt * (I.dt ? *I.dt : 0.0);
    const double X = I.U_inf * time / I.L;
    const double* md = I.modes + c * 4 * nm;
    for (int t = threadIdx.x; t < nr * nm; t += IN_EXT_NT) {
        const int rr = t / nm, q = t - rr * nm;
        const int row = r0 + rr, m = row / Nj, j = row - m * Nj, gi = ng - 1 - m;
        const double y = B.met[WM_MET_XCY * B.ncell + ((long long)gi * Nj + j) * Nk] / I.L;
        double s_, c_;
        sincos((md[q] * X + md[nm + q] * y) + md[3 * nm + q], &s_, &c_);
        ta[(2 * rr) * nm + q] = c_;
        ta[(2 * rr + 1) * nm + q] = s_;
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    for (int t = threadIdx.x; t < nr * Nk; t += IN_EXT_NT) {
        const int rr = t / Nk, k = t - rr * Nk;
        const double* ca = ta + 2 * rr * nm;
        const double* sa = ca + nm;
        double a0 = 0.0, a1 = 0.0;          // even and odd modes
        int q = 0;
        for (; q + 1 < nm; q += 2) {
            a0 += ca[q] * tb[q * Nk + k] - sa[q] * tb[(nm + q) * Nk + k];
            a1 += ca[q + 1] * tb[(q + 1) * Nk + k] - sa[q + 1] * tb[(nm + q + 1) * Nk + k];
        }
        if (q < nm) a0 += ca[q] * tb[q * Nk + k] - sa[q] * tb[(nm + q) * Nk + k];
        I.raw[((long long)(r0 + rr) * 3 + c) * Nk + k] = a0 + a1;
    }
}

// one ghost row (layer m, j) of any plane: the raw mode sums (parts ranges, added in range
// order), the row's normalisation of wmles/smooth_ramp.py:186-196 by warp c for component c
// (warp sums; component 1 takes component 0's final values after a barrier), the ghost states
__global__ void __launch_bounds__(IN_ROW_NT) inflow_row_kernel(const __grid_constant__ InflowArgs I, int parts) {
    extern __shared__ double sm[];          // noise: 3 x Nk
    const BlockDev& B = *I.block;
    const int ng = B.ng, Nj = B.N[1], Nk = B.N[2], nk = B.n[2];
    const int j = blockIdx.x, m = blockIdx.y, gi = ng - 1 - m;
    const int c = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long rows = (long long)ng * Nj, row = (long long)m * Nj + j;
    double* f = sm + c * Nk;
    for (int k = lane; k < Nk; k += 32) {
        double acc = I.raw[(row * 3 + c) * Nk + k];
        for (int pt = 1; pt < parts; ++pt) acc += I.raw[((pt * rows + row) * 3 + c) * Nk + k];
        f[k] = acc;
    }
    __syncwarp();
    double s_int = 0.0;
    for (int k = ng + lane; k < ng + nk; k += 32) s_int += f[k];
    const double mean = warp_allsum(s_int) / nk;
    for (int k = lane; k < Nk; k += 32) f[k] -= mean;
    __syncwarp();
    auto normalise = [&]() {
        double v_acc = 0.0;
        for (int k = ng + lane; k < ng + nk; k += 32) v_acc += f[k] * f[k];
        const double inv = 1.0 / sqrt(fmax(warp_allsum(v_acc) / nk, 1e-20));
        for (int k = lane; k < Nk; k += 32) f[k] *= inv;
    };
    if (c != 1) normalise();
    __syncthreads();
    if (c == 1) {
        const double* f0 = sm;
        double cov_acc = 0.0;
        for (int k = ng + lane; k < ng + nk; k += 32) cov_acc += f[k] * f0[k];
        const double cov = warp_allsum(cov_acc) / nk;
        for (int k = lane; k < Nk; k += 32) f[k] -= cov * f0[k];
        __syncwarp();
        normalise();
    }
    __syncthreads();
    const long long row0 = ((long long)gi * Nj + j) * Nk;
    for (int k = threadIdx.x; k < Nk; k += IN_ROW_NT)
        inflow_write(I, row0 + k, (long long)ng * Nj * Nk, sm[k], sm[Nk + k], sm[2 * Nk + k]);
}

cudaError_t launch_inflow_setup(const InflowArgs& I, int Nj, int Nk, int ng, double* prof, double* cz, cudaStream_t s) {
    const long long n = (long long)ng * Nj * Nk;
    inflow_prof_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(I, prof, n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || cz == nullptr) return e;
    const int t = 3 * I.n_modes * Nk;
    inflow_cz_kernel<<<(t + 255) / 256, 256, 0, s>>>(I, Nk, cz);
    return cudaGetLastError();
}

size_t inflow_ext_smem(int n_modes, int Nk) {
    return sizeof(double) * (2 * (size_t)n_modes * Nk + 2 * (size_t)IN_EXT_ROWS * n_modes);
}

cudaError_t launch_inflow(const InflowArgs& I, int Nj, int Nk, int ng, cudaStream_t s) {
    int parts = IN_PARTS;
    if (I.cz != nullptr) {
        const size_t sm = inflow_ext_smem(I.n_modes, Nk);
        static std::atomic<unsigned long long> attr{0};     // one bit per device
        const cudaError_t e = once_per_device(attr, [] {
            return cudaFuncSetAttribute(inflow_ext_sums_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)inflow_ext_smem_max());
        });
        if (e != cudaSuccess) return e;
        inflow_ext_sums_kernel<<<dim3((ng * Nj + IN_EXT_ROWS - 1) / IN_EXT_ROWS, 3), IN_EXT_NT, sm, s>>>(I);
        parts = 1;
    } else {
        const long long units = (long long)IN_PARTS * ng * Nj * 3 * Nk;
        inflow_modes_kernel<<<(unsigned)((units + IN_NT - 1) / IN_NT), IN_NT, 0, s>>>(I, units);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    inflow_row_kernel<<<dim3(Nj, ng), IN_ROW_NT, sizeof(double) * 3 * Nk, s>>>(I, parts);
    return cudaGetLastError();
}

}  // namespace wm
