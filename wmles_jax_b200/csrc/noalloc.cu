// CFL time step without any device allocation (wm_max_dt_noalloc, include/wmles_cuda.h).
//
// For callers that cannot allocate device memory at all: code that runs inside another
// framework's memory pool (a JAX/XLA custom call or a PyTorch extension that must not
// bypass the caching allocator), a CUDA-graph node added by someone else, or a process
// with a hard device-memory budget.  The caller passes the state, the metrics and the
// output slot; the only scratch the reduction needs (one partial minimum per CTA and a
// done-counter) lives in the file-scope array below, which every GPU that loads this
// library holds until the process exits.
//
// Each call clears the counter on its stream before the kernel, and the kernel's last
// CTA clears it again.  The array is shared by every call: calls that overlap on the GPU
// (different streams, or threads issuing concurrently) race on it and must be serialised
// by the caller.
#include <cstdio>
#include <mutex>
#include <cuda.h>              // CUcontext / CUresult types only: the driver calls are looked up
#include "wm_internal.cuh"

namespace {

constexpr int kMaxDevices = 64;
constexpr int kThreads = 256;

// [0]: done-counter, [1 .. WM_NOALLOC_MAX_PARTIALS]: per-CTA minima (double bit patterns)
static __device__ __align__(256) unsigned long long g_noalloc_scratch[1 + WM_NOALLOC_MAX_PARTIALS];

// per device: the scratch array's address and the id of the context it was looked up in
// (a context destroyed by cudaDeviceReset and created again reloads the module, possibly
// elsewhere, so the address is looked up again when the id changes)
unsigned long long* g_scratch_addr[kMaxDevices] = {nullptr};
unsigned long long g_scratch_ctx[kMaxDevices] = {0};
std::mutex g_scratch_mutex;

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;

struct NoAllocArgs {
    int nblocks, total_ctas;
    int cta_start[WM_MAX_BLOCKS + 1];
    int dims[WM_MAX_BLOCKS][4];          // ni, nj, nk, ng
    const double* q[WM_MAX_BLOCKS];
    const double* met[WM_MAX_BLOCKS];
    double gamma, Rg, gm1, mu_ref, inv_Tref, TrefS, S_suth, nu_fac, cfl;
    unsigned long long* scratch;
    double* dt_out;
};

__device__ __forceinline__ double nanmin_d(double a, double b) { return (a != a || a < b) ? a : b; }

// Solver._dt (wmles/solver.py:135-151) on interior cells, one cell per thread
__global__ void __launch_bounds__(kThreads) cfl_noalloc_kernel(const __grid_constant__ NoAllocArgs A) {
    __shared__ double red[kThreads / 32];
    __shared__ bool last;
    const int cta = blockIdx.x;
    int b = 0;
    while (b + 1 < A.nblocks && cta >= A.cta_start[b + 1]) ++b;
    const int ni = A.dims[b][0], nj = A.dims[b][1], nk = A.dims[b][2], ng = A.dims[b][3];
    const long long Nj = nj + 2 * ng, Nk = nk + 2 * ng;
    const long long plane = Nj * Nk, N = plane * (ni + 2 * ng);
    const long long c = (long long)(cta - A.cta_start[b]) * kThreads + threadIdx.x;
    double dt = 1.7976931348623157e308;
    if (c < (long long)ni * nj * nk) {
        const int i = int(c / ((long long)nj * nk)) + ng;
        const int r = int(c % ((long long)nj * nk));
        const long long idx = i * plane + (long long)(r / nk + ng) * Nk + (r % nk + ng);
        const double* q = A.q[b];
        const double* met = A.met[b];
        const double rho = q[idx];
        const double ir = 1.0 / rho;
        const double u = q[N + idx] * ir, v = q[2 * N + idx] * ir, w = q[3 * N + idx] * ir;
        const double p = A.gm1 * (q[4 * N + idx] - 0.5 * rho * ((u * u + v * v) + w * w));
        const double T = p * ir / A.Rg;
        const double x = T * A.inv_Tref;
        const double nu = A.nu_fac * (A.mu_ref * (x * sqrt(x)) * A.TrefS / (T + A.S_suth)) * ir;
        const double cs = sqrt(A.gamma * A.Rg * T);
        const double vol = met[WM_MET_VOL * N + idx];
        const long long off[3] = {plane, Nk, 1};
        double lam = 0.0, lamv = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double* S = met + 3 * d * N;
            const double sx = 0.5 * (S[idx] + S[idx + off[d]]);
            const double sy = 0.5 * (S[N + idx] + S[N + idx + off[d]]);
            const double sz = 0.5 * (S[2 * N + idx] + S[2 * N + idx + off[d]]);
            const double Sm = sqrt((sx * sx + sy * sy) + sz * sz);
            lam = lam + fabs((u * sx + v * sy) + w * sz) + cs * Sm;
            lamv = lamv + nu * (Sm * Sm) / vol;
        }
        dt = A.cfl / ((lam + 4.0 * lamv) / vol);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dt = nanmin_d(dt, __shfl_down_sync(0xffffffffu, dt, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dt;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
        for (int k = 1; k < kThreads / 32; ++k) m = nanmin_d(m, red[k]);
        A.scratch[1 + cta] = static_cast<unsigned long long>(__double_as_longlong(m));
        __threadfence();
        last = atomicAdd(&A.scratch[0], 1ull) == static_cast<unsigned long long>(A.total_ctas - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double m = 1.7976931348623157e308;
    const volatile unsigned long long* part = A.scratch + 1;
    for (int k = threadIdx.x; k < A.total_ctas; k += kThreads) m = nanmin_d(m, __longlong_as_double((long long)part[k]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = nanmin_d(m, __shfl_down_sync(0xffffffffu, m, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double mm = red[0];
        for (int k = 1; k < kThreads / 32; ++k) mm = nanmin_d(mm, red[k]);
        *A.dt_out = mm;
        A.scratch[0] = 0ull;
    }
}

int fail(int code, const char* msg) { return wm::set_error(code, msg); }

// id of the calling thread's current context (0: none current yet), through driver entry
// points looked up once (the library does not link the driver library itself)
unsigned long long current_context_id() {
    if (!g_ctx_current || !g_ctx_id) {
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", (void**)&g_ctx_current, 12000, cudaEnableDefault, &q1) !=
                cudaSuccess || q1 != cudaDriverEntryPointSuccess ||
            cudaGetDriverEntryPointByVersion("cuCtxGetId", (void**)&g_ctx_id, 12000, cudaEnableDefault, &q2) !=
                cudaSuccess || q2 != cudaDriverEntryPointSuccess) {
            g_ctx_current = nullptr;
            g_ctx_id = nullptr;
            return 0;
        }
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (g_ctx_current(&ctx) != CUDA_SUCCESS || ctx == nullptr || g_ctx_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// device address of the scratch array on the current device: looked up once per device and
// context (at the first call, and again after the device's context was replaced)
int scratch_address(unsigned long long** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(WM_E_CUDA, "wm_max_dt_noalloc: no usable current device");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    const unsigned long long ctx = current_context_id();
    if (g_scratch_addr[dev] == nullptr || ctx == 0 || ctx != g_scratch_ctx[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            char m[200];
            snprintf(m, sizeof(m), "wm_max_dt_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return fail(WM_E_CUDA, m);
        }
        g_scratch_addr[dev] = static_cast<unsigned long long*>(p);
        g_scratch_ctx[dev] = current_context_id();     // the lookup made the context current
    }
    *out = g_scratch_addr[dev];
    return WM_OK;
}

}  // namespace

extern "C" {

int wm_max_dt_noalloc(int nblocks, const int* dims, const double* const* q, const double* const* metrics,
                      const wm_gas* gas, double cfl, double* dt_dev, void* stream) {
    if (nblocks < 1 || nblocks > WM_MAX_BLOCKS || !dims || !q || !metrics || !gas || !dt_dev)
        return fail(WM_E_INVALID, "wm_max_dt_noalloc: bad arguments (nblocks in [1, WM_MAX_BLOCKS], non-null pointers)");
    NoAllocArgs A{};
    A.nblocks = nblocks;
    long long total = 0;
    for (int b = 0; b < nblocks; ++b) {
        for (int x = 0; x < 4; ++x) A.dims[b][x] = dims[4 * b + x];
        if (A.dims[b][3] < 1 || A.dims[b][0] < A.dims[b][3] || A.dims[b][1] < A.dims[b][3] || A.dims[b][2] < A.dims[b][3])
            return fail(WM_E_INVALID, "wm_max_dt_noalloc: each block needs ng >= 1 and at least ng cells per direction");
        if (!q[b] || !metrics[b]) return fail(WM_E_INVALID, "wm_max_dt_noalloc: null state or metrics pointer");
        A.q[b] = q[b];
        A.met[b] = metrics[b];
        A.cta_start[b] = (int)total;
        total += ((long long)A.dims[b][0] * A.dims[b][1] * A.dims[b][2] + kThreads - 1) / kThreads;
        if (total > WM_NOALLOC_MAX_PARTIALS) {
            char m[200];
            snprintf(m, sizeof(m), "wm_max_dt_noalloc: the blocks need %lld reduction slots, the static scratch holds %d "
                     "(at most %d interior cells in total)", total, WM_NOALLOC_MAX_PARTIALS,
                     WM_NOALLOC_MAX_PARTIALS * kThreads);
            return fail(WM_E_INVALID, m);
        }
    }
    A.cta_start[nblocks] = (int)total;
    A.total_ctas = (int)total;
    A.gamma = gas->gamma; A.Rg = gas->R; A.gm1 = gas->gamma - 1.0; A.mu_ref = gas->mu_ref;
    A.inv_Tref = 1.0 / gas->T_ref; A.TrefS = gas->T_ref + gas->S_suth; A.S_suth = gas->S_suth;
    A.nu_fac = gas->gamma / gas->Pr > 4.0 / 3.0 ? gas->gamma / gas->Pr : 4.0 / 3.0;
    A.cfl = cfl;
    A.dt_out = dt_dev;
    int r = scratch_address(&A.scratch);
    if (r) return r;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(A.scratch, 0, sizeof(unsigned long long), s);    // done-counter = 0
    if (e == cudaSuccess) {
        cfl_noalloc_kernel<<<A.total_ctas, kThreads, 0, s>>>(A);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        char m[200];
        snprintf(m, sizeof(m), "wm_max_dt_noalloc: %s", cudaGetErrorString(e));
        return fail(WM_E_CUDA, m);
    }
    return WM_OK;
}

}  // extern "C"
