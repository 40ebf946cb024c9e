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
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/pgmg_dev.h"

namespace {

constexpr int kNaBlock = 256;
constexpr long kNaMaxBlocks = 65536;                  // at most 65536 * 256 = 16,777,216 points
constexpr long kNaMaxPoints = kNaMaxBlocks * kNaBlock;
constexpr int kNaMaxDevices = 64;

// Per-block partial sums (sum res^2, sum r^2), 1 MiB per device.
static __device__ __align__(256) double g_na_partials[2 * kNaMaxBlocks];

// Device address of g_na_partials, looked up once per device.
double* g_na_ptr[kNaMaxDevices] = {};
std::mutex g_na_mu;

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
    long npts = (long)m * n * o;
    if (npts > kNaMaxPoints) return PGMG_ERR_ARG;  // beyond the fixed scratch: 2^24 points
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return PGMG_ERR_NO_DEVICE;
    }
    if (dev < 0 || dev >= kNaMaxDevices) return PGMG_ERR_UNSUPPORTED;
    if (!on_device(coef27, dev) || !on_device(x, dev) || !on_device(r, dev) || !on_device(out, dev))
        return PGMG_ERR_ARG;
    double* part = nullptr;
    {
        // First call on this device: the address of the fixed array, with
        // this device current.
        std::lock_guard<std::mutex> lk(g_na_mu);
        if (!g_na_ptr[dev]) {
            double* p = nullptr;
            if (cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_na_partials) != cudaSuccess || !p) {
                cudaGetLastError();
                return PGMG_ERR_CUDA;
            }
            g_na_ptr[dev] = p;
        }
        part = g_na_ptr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    long nb = (npts + kNaBlock - 1) / kNaBlock;
    k_na_partials<<<(unsigned)nb, kNaBlock, 0, s>>>(m, n, o, coef27, x, r, part);
    k_na_reduce<<<1, 1024, 0, s>>>(part, nb, out);
    if (cudaGetLastError() != cudaSuccess) return PGMG_ERR_CUDA;
    return PGMG_OK;
}
