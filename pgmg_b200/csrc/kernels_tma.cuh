// The 8-colour pass with its stencil coefficients and sources staged in
// shared memory by the Tensor Memory Accelerator (cp.async.bulk), an
// autotuned alternative to k_gs_colour / k_gs_colour_pf on non-periodic
// levels swept in one slab.
//
// A CTA of BS threads owns BS consecutive colour points of one colour.  In
// the colour-major layout each of their 27 stencil slots is one contiguous
// run of BS values in its slot plane, and so is their source: one thread
// issues 28 bulk copies (global -> shared, one per run) that complete on one
// mbarrier, the 27 stencil runs before the kernel waits for the previous one
// (stencils are written only at set-up, so they can be fetched while that
// kernel drains) and the source run after.  The whole stencil stream is then
// in flight per CTA with no register cost; the threads read their
// coefficients from shared memory and the neighbours' x from L2 as
// k_gs_colour does, with the same arithmetic, so the pass is bit-identical.
//
// Alignment: slot planes start on 256-byte boundaries (Nc is a multiple of
// 64) and a CTA's first point is a multiple of BS (>= 64), so every copy
// starts on a 16-byte boundary; the last CTA's runs are rounded up to 16
// bytes, which stays inside the plane's padding (Nc >= the point count
// rounded up to 64).  No tensor map and no multicast is used.
//
// The mbarrier wait is bounded (kTmaWaitCycles of the SM clock, about half a
// second): a wait that runs out sets the error word, waits once more, as
// long, for the CTA's own copies, and returns; the host reports
// PGMG_ERR_TIMEOUT.  `extra_tx` (0 in use) makes the barrier expect more
// bytes than are copied, so that a self-check can make the wait run out.
#pragma once
#include "layout.cuh"

namespace pgmg {

constexpr long long kTmaWaitCycles = 1LL << 30;

__device__ __forceinline__ uint32_t tma_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tma_smem_u32(bar)), "r"(count) : "memory");
}
// Makes the initialised barrier visible to the asynchronous (TMA) proxy.
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tma_smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// Bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned)
// from global to this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     tma_smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(tma_smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(tma_smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the completion of the barrier phase with `parity`, for at most
// kTmaWaitCycles; false if it ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
    long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > kTmaWaitCycles) return false;
    return true;
}

template <class T, int BS>
constexpr size_t gs_tma_smem() {
    return 28 * BS * sizeof(T) + 16;
}

template <class T, int BS>
__global__ void __launch_bounds__(BS) k_gs_colour_tma(LevelGeom g, T* x, const T* __restrict__ r,
                                                      const T* __restrict__ A, int col, int rev, int* err,
                                                      unsigned extra_tx) {
    extern __shared__ __align__(128) unsigned char tma_raw[];
    T* sa = reinterpret_cast<T*>(tma_raw);  // [28][BS]: slots 0..26, then the source
    uint64_t* bar = reinterpret_cast<uint64_t*>(tma_raw + 28 * BS * sizeof(T));
    const long nc = (long)g.M2 * g.N2 * g.O2;
    const unsigned b = rev ? gridDim.x - 1 - blockIdx.x : blockIdx.x;
    const long p0 = (long)b * BS;
    const long L = nc - p0 < BS ? nc - p0 : BS;
    const unsigned run = (unsigned)((L * (long)sizeof(T) + 15) & ~15L);
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect_tx(bar, 28u * run + extra_tx);
        const T* Ap = A + (long)col * 27 * g.Nc + p0;
        for (int q = 0; q < 27; q++) bulk_g2s(sa + q * BS, Ap + q * g.Nc, run, bar);
    }
    pdl_enter();
    if (threadIdx.x == 0) bulk_g2s(sa + 27 * BS, r + (long)col * g.Nc + p0, run, bar);
    if (!mbar_wait_bounded(bar, 0)) {
        if (threadIdx.x == 0) atomicExch(err, 1);
        mbar_wait_bounded(bar, 0);  // the CTA's own copies, before its shared memory goes
        return;
    }
    const long p = p0 + threadIdx.x;
    if (p >= nc) return;
    int i2, j2, k2;
    decode_colour(g, p, i2, j2, k2);
    const int i = 2 * i2 + (col & 1), j = 2 * j2 + ((col >> 1) & 1), k = 2 * k2 + (col >> 2);
    if (i >= g.m || j >= g.n || k >= g.o) return;
    const uint64_t pk = policy_evict_last();
    const long xc = g.xi(i, j, k);
    const T* sp = sa + threadIdx.x;
    T acc = T(0);
#pragma unroll
    for (int q = 0; q < 27; q++) {
        if (q == 13) continue;
        acc = madd<true, T>(acc, sp[q * BS], ld_keep(x + xc + slot_off(g, q), pk));
    }
    st_keep(x + xc, mul_rn<T>(sub_rn<T>(sp[27 * BS], acc), T(1) / sp[13 * BS]), pk);
}

}  // namespace pgmg
