// Residual norms without any device allocation.
//
// Some callers cannot allocate device memory: a host framework that owns the
// whole card through its own memory pool and forbids other allocations, or a
// latency-critical loop in which a cudaMalloc/cudaFree would stall or
// synchronise the device.  For them, pgmg_residual_norms_noalloc computes
// sum (r - A x)^2 and sum r^2 of a 27-point operator from caller-owned device
// arrays, and keeps its only intermediate data -- one pair of partial sums per
// thread block -- in a fixed array of this file that every GPU loading the
// library holds until the process exits.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/pgmg_dev.h"

namespace {

constexpr int kNaBlock = 256;
constexpr long kNaMaxBlocks = 65536;                  // at most 65536 * 256 = 16,777,216 points
constexpr long kNaMaxPoints = kNaMaxBlocks * kNaBlock;
constexpr int kNaMaxContexts = 64;

// Per-block partial sums (sum res^2, sum r^2), 1 MiB per device.
static __device__ __align__(256) double g_na_partials[2 * kNaMaxBlocks];

// Device address of g_na_partials per CUDA context.  The array's address
// belongs to the context the module was loaded in: a caller that switches
// to another context (its own cuCtxCreate context, or the primary context
// re-created after cudaDeviceReset) gets a fresh look-up, never an address
// of a context that is gone or not current.
struct NaEntry {
    CUcontext ctx;
    double* ptr;
};
NaEntry g_na_cache[kNaMaxContexts] = {};
int g_na_used = 0;
std::mutex g_na_mu;

// cuCtxGetCurrent through the runtime's driver entry point, so that the
// library needs no link-time dependency on the driver library.
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {
    static CtxGetCurrentFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

__device__ __forceinline__ void na_sum2(double& a, double& b, double* sh) {
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (l == 0) { sh[w] = a; sh[32 + w] = b; }
    __syncthreads();
    if (w == 0) {
        a = l < nw ? sh[l] : 0.0;
        b = l < nw ? sh[32 + l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
    }
}

// One thread per grid point (natural order): the residual summed over the 27
// slots in box order, each product and sum rounded separately (the order of
// the reference's region::residual); slots that reach outside the grid are
// skipped.  Every block writes its pair of partial sums.
__global__ void __launch_bounds__(kNaBlock) k_na_partials(int m, int n, int o, const double* __restrict__ c27,
                                                         const double* __restrict__ x, const double* __restrict__ r,
                                                         double* __restrict__ partials) {
    __shared__ double sh[64];
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long npts = (long)m * n * o;
    double s_res = 0, s_rhs = 0;
    if (q < npts) {
        int i = (int)(q % m);
        long t = q / m;
        int j = (int)(t % n);
        int k = (int)(t / n);
        const double* c = c27 + 27 * q;
        double acc = 0.0;
        for (int s = 0; s < 27; s++) {
            int ii = i + s % 3 - 1, jj = j + (s / 3) % 3 - 1, kk = k + s / 9 - 1;
            if (ii < 0 || jj < 0 || kk < 0 || ii >= m || jj >= n || kk >= o) continue;
            acc = __dadd_rn(acc, __dmul_rn(c[s], x[ii + (long)m * (jj + (long)n * kk)]));
        }
        double rv = r[q];
        double res = __dsub_rn(rv, acc);
        s_res = res * res;
        s_rhs = rv * rv;
    }
    na_sum2(s_res, s_rhs, sh);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = s_res;
        partials[2 * blockIdx.x + 1] = s_rhs;
    }
}

__global__ void __launch_bounds__(1024) k_na_reduce(const double* __restrict__ partials, long nb,
                                                    double* __restrict__ out) {
    __shared__ double sh[64];
    double a = 0, b = 0;
    for (long q = threadIdx.x; q < nb; q += blockDim.x) {
        a += partials[2 * q];
        b += partials[2 * q + 1];
    }
    na_sum2(a, b, sh);
    if (threadIdx.x == 0) {
        out[0] = a;
        out[1] = b;
    }
}

bool on_device(const void* p, int dev) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
}

}  // namespace

extern "C" pgmg_status pgmg_residual_norms_noalloc(int m, int n, int o, const double* coef27, const double* x,
                                                   const double* r, double* out, void* stream) {
    if (m < 1 || n < 1 || o < 1 || !coef27 || !x || !r || !out) return PGMG_ERR_ARG;
    // Beyond the fixed scratch (2^24 points): each partial product is
    // bounded before the next multiplication, so no product can overflow.
    if (m > kNaMaxPoints || (long)m * n > kNaMaxPoints || (long)m * n * o > kNaMaxPoints) return PGMG_ERR_ARG;
    long npts = (long)m * n * o;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return PGMG_ERR_NO_DEVICE;
    }
    if (!on_device(coef27, dev) || !on_device(x, dev) || !on_device(r, dev) || !on_device(out, dev))
        return PGMG_ERR_ARG;
    CtxGetCurrentFn get_ctx = ctx_get_current();
    if (!get_ctx) return PGMG_ERR_UNSUPPORTED;
    double* part = nullptr;
    {
        // The address of the fixed array in the current context, looked up
        // with that context current on its first call there.
        std::lock_guard<std::mutex> lk(g_na_mu);
        CUcontext ctx = nullptr;
        if (get_ctx(&ctx) != CUDA_SUCCESS || !ctx) return PGMG_ERR_CUDA;
        for (int e = 0; e < g_na_used && !part; e++)
            if (g_na_cache[e].ctx == ctx) part = g_na_cache[e].ptr;
        if (!part) {
            double* p = nullptr;
            if (cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_na_partials) != cudaSuccess || !p) {
                cudaGetLastError();
                return PGMG_ERR_CUDA;
            }
            // A full table recycles its oldest entry.
            int e = g_na_used < kNaMaxContexts ? g_na_used++ : 0;
            if (e == 0 && g_na_used == kNaMaxContexts) {
                for (int q = 1; q < kNaMaxContexts; q++) g_na_cache[q - 1] = g_na_cache[q];
                e = kNaMaxContexts - 1;
            }
            g_na_cache[e] = {ctx, p};
            part = p;
        }
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    long nb = (npts + kNaBlock - 1) / kNaBlock;
    k_na_partials<<<(unsigned)nb, kNaBlock, 0, s>>>(m, n, o, coef27, x, r, part);
    k_na_reduce<<<1, 1024, 0, s>>>(part, nb, out);
    if (cudaGetLastError() != cudaSuccess) return PGMG_ERR_CUDA;
    return PGMG_OK;
}
