// Persistent whole-GPU sweeps of a mid-sized level.
//
// A level of a few hundred thousand to a few million points is swept by 8 x
// (2+l) colour passes per V-cycle leg; as separate launches each pass pays
// a launch ramp and drain that is as long as its work.  k_sweeps_grid runs
// every colour pass of a leg's sweeps in ONE cooperative launch (all blocks
// co-resident), the passes separated by a software grid barrier.
//
// The barrier is a counter and a generation word in global memory.  Its
// spin is bounded: a block that waits longer than kGridSpinLimit polls (about
// a second) sets the error word and leaves, every other block leaves at its
// next barrier when it sees the error, and the host reports PGMG_ERR_TIMEOUT
// -- the kernel never hangs the GPU.
//
// x is written by one pass and read by other blocks in the next, so it is
// loaded with ld.global.cg (L2, never a stale L1 or non-coherent-cache
// line); stencils and sources are read-only for the kernel and use the same
// streaming loads as k_gs_colour.  The arithmetic is gs_value's, so the
// sweeps are bit-identical to the per-pass launches.
#pragma once
#include "layout.cuh"

namespace pgmg {

struct GridBar {
    unsigned count;  // blocks arrived at the current barrier
    unsigned gen;    // barriers completed
    int err;         // 1: a wait ran out
    int tma_err;     // 1: an mbarrier wait of the TMA colour pass (k_gs_colour_tma) ran out
};

constexpr long kGridSpinLimit = 1L << 21;

__device__ __forceinline__ double ld_l2(const double* a) { return __ldcg(a); }
__device__ __forceinline__ float ld_l2(const float* a) { return __ldcg(a); }

// All blocks of the grid meet; false if the barrier failed (a wait ran out).
__device__ __forceinline__ bool grid_sync(GridBar* b, unsigned nblocks) {
    __syncthreads();
    __shared__ int ok;
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = &b->gen;
        volatile int* verr = &b->err;
        unsigned g0 = *vgen;
        int good = *verr == 0;
        __threadfence();  // this block's writes before its arrival
        if (good) {
            if (atomicAdd(&b->count, 1u) == nblocks - 1) {
                atomicExch(&b->count, 0u);
                __threadfence();
                atomicAdd(&b->gen, 1u);
            } else {
                long spins = 0;
                while (*vgen == g0) {
                    if (*verr) { good = 0; break; }
                    if (++spins > kGridSpinLimit) {
                        atomicExch(&b->err, 1);
                        good = 0;
                        break;
                    }
                    __nanosleep(64);
                }
            }
        }
        __threadfence();  // the other blocks' writes after the barrier
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

template <class T>
__device__ __forceinline__ void gs_point_l2(const LevelGeom& g, T* x, const T* __restrict__ r,
                                            const T* __restrict__ A, int col, long p, uint64_t ps, uint64_t pk) {
    int i2, j2, k2;
    decode_colour(g, p, i2, j2, k2);
    int i = 2 * i2 + (col & 1), j = 2 * j2 + ((col >> 1) & 1), k = 2 * k2 + (col >> 2);
    if (i >= g.m || j >= g.n || k >= g.o) return;
    long xc = g.xi(i, j, k);
    const T* Ap = A + (long)col * 27 * g.Nc + p;
    T acc = T(0);
#pragma unroll
    for (int q = 0; q < 27; q++) {
        if (q == 13) continue;
        acc = madd<true, T>(acc, ld_stream(Ap + q * g.Nc, ps), ld_l2(x + xc + slot_off(g, q)));
    }
    T inv = T(1) / ld_stream(Ap + 13 * g.Nc, ps);
    T v = mul_rn<T>(sub_rn<T>(ld_stream(r + (long)col * g.Nc + p, ps), acc), inv);
    st_keep(x + xc, v, pk);
}

// `sweeps` sweeps (forward colour order, then backward when mode != 0) of a
// non-periodic level, one slab.  Launched cooperatively with at most as many
// blocks as fit on the GPU at once.
// `expect`: the blocks a barrier waits for -- gridDim.x, except in the
// self-check that makes a wait run out on purpose (gridDim.x + 1).
template <class T>
__global__ void __launch_bounds__(512, 2) k_sweeps_grid(LevelGeom g, T* x, const T* __restrict__ r,
                                                        const T* __restrict__ A, int sweeps, int mode,
                                                        GridBar* bar, unsigned expect) {
    long nc = (long)g.M2 * g.N2 * g.O2;
    long stride = (long)gridDim.x * blockDim.x;
    uint64_t ps = policy_evict_first(), pk = policy_evict_last();
    int per = mode ? 16 : 8, total = sweeps * per;
    for (int st = 0; st < total; st++) {
        int cc = st % per;
        int col = colour_seq(cc < 8 ? cc : 15 - cc);
        for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < nc; p += stride)
            gs_point_l2<T>(g, x, r, A, col, p, ps, pk);
        if (st + 1 < total && !grid_sync(bar, expect)) return;
    }
}

}  // namespace pgmg
