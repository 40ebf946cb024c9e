// Hot-path kernels: Gauss-Seidel smoothers, residual (+norms), restriction,
// interpolation, field movement.  All templated on the storage type T
// (double for the FP64 V-cycle, float for the FP32 V-cycle of mixed
// precision); EXACT selects reference-order arithmetic without fused
// multiply-add (bitwise parity with the reference's x86-64 build).
#pragma once
#include "layout.cuh"

namespace pgmg {

constexpr int kBlock = 256;

// ---------------------------------------------------------------------------
// Gauss-Seidel point update (region.cc:367-446): terms in box order with the
// centre skipped, x = (r - Ax) * (1/centre).  Stencil slots outside the box
// are zero, so summing all 26 in slot order is the reference's box order.
template <class T, bool EXACT>
__device__ __forceinline__ T gs_value(const LevelGeom& g, const T* __restrict__ x, long xc,
                                      const T* __restrict__ Ap, long plane, T rv, uint64_t pstream,
                                      uint64_t pkeep) {
    T acc = T(0);
#pragma unroll
    for (int q = 0; q < 27; q++) {
        if (q == 13) continue;
        acc = madd<EXACT, T>(acc, ld_stream(Ap + q * plane, pstream), ld_keep(x + xc + slot_off(g, q), pkeep));
    }
    T inv = T(1) / ld_stream(Ap + 13 * plane, pstream);
    if (EXACT) return mul_rn<T>(sub_rn<T>(rv, acc), inv);
    return (rv - acc) * inv;
}

// K1: one colour of the 8-colour sweep.  Points of one colour are mutually
// independent for a 27-point box, so the colour is one fully parallel pass;
// the 26 neighbours read here belong to other colours and are not written
// by this launch.  One thread per colour point; coefficient slot q of
// consecutive threads is contiguous (structure-of-arrays per colour).
// One colour point p (index inside colour `col`): the body of k_gs_colour,
// shared with the batched kernels.
template <class T, bool PRD = false>
__device__ __forceinline__ void gs_colour_at(const LevelGeom& g, T* x, const T* __restrict__ r,
                                             const T* __restrict__ A, int col, long p) {
    int i2, j2, k2;
    decode_colour(g, p, i2, j2, k2);
    int i = 2 * i2 + (col & 1), j = 2 * j2 + ((col >> 1) & 1), k = 2 * k2 + (col >> 2);
    if (i >= g.m || j >= g.n || k >= g.o) return;
    uint64_t ps = policy_evict_first(), pk = policy_evict_last();
    long xc = g.xi(i, j, k);
    const T* Ap = A + (long)col * 27 * g.Nc + p;
    T v = gs_value<T, true>(g, x, xc, Ap, g.Nc, ld_stream(r + (long)col * g.Nc + p, ps), ps, pk);
    st_keep(x + xc, v, pk);
    // Periodic axes (PRD: a separate instantiation, so that the usual one
    // keeps its register count): the point's images in the halo are updated
    // with it; the points that read them are of other colours (periodic sizes
    // are even).
    if (PRD) store_images<T>(g, x, i, j, k, v);
}

// BS: threads per block (the autotuner picks 128, 256 or 512 per handle).
// rev: blocks take the points from the top (last z planes) down.  Blocks
// are scheduled in index order, so a pass with rev = 1 starts where the
// previous pass ended and reads the solution planes that pass left in L2;
// the points of one colour are independent, so the order changes no result.
template <class T, bool EXACT, bool PRD = false, int BS = kBlock>
__global__ void __launch_bounds__(BS) k_gs_colour(LevelGeom g, T* x, const T* __restrict__ r,
                                                      const T* __restrict__ A, int col, int k2lo, int k2hi,
                                                      int rev) {
    pdl_enter();
    unsigned b = rev ? gridDim.x - 1 - blockIdx.x : blockIdx.x;
    long p = (long)k2lo * g.M2 * g.N2 + b * (long)blockDim.x + threadIdx.x;
    if (p >= (long)k2hi * g.M2 * g.N2) return;
    gs_colour_at<T, PRD>(g, x, r, A, col, p);
}

// The same colour pass with 16-byte vector loads: each thread updates V =
// 16/sizeof(T) consecutive colour points (2 FP64, 4 FP32), loading the V
// points' coefficient of each stencil slot, their sources and diagonals with
// one 128-bit load each.  Every point's arithmetic is gs_value's, in the same
// order, so results are bit-identical to k_gs_colour.  One slab only (p
// starts at 0, so every thread's first point is a multiple of V and its loads
// are aligned: colour-major planes are padded to multiples of 64 points).
template <class T, int BS, int V = 16 / sizeof(T)>
__global__ void __launch_bounds__(BS) k_gs_colour_v(LevelGeom g, T* x, const T* __restrict__ r,
                                                    const T* __restrict__ A, int col, int rev) {
    pdl_enter();
    long nc = (long)g.M2 * g.N2 * g.O2;
    unsigned b = rev ? gridDim.x - 1 - blockIdx.x : blockIdx.x;
    long p0 = (b * (long)BS + threadIdx.x) * V;
    if (p0 >= nc) return;
    uint64_t ps = policy_evict_first(), pk = policy_evict_last();
    const long safe = g.xi(0, 0, 0);  // a point whose 27 neighbours exist (halo)
    long xc[V];
    bool ok[V];
#pragma unroll
    for (int v = 0; v < V; v++) {
        int i2, j2, k2;
        decode_colour(g, p0 + v, i2, j2, k2);
        int i = 2 * i2 + (col & 1), j = 2 * j2 + ((col >> 1) & 1), k = 2 * k2 + (col >> 2);
        ok[v] = p0 + v < nc && i < g.m && j < g.n && k < g.o;
        xc[v] = ok[v] ? g.xi(i, j, k) : safe;
    }
    const T* Ap = A + (long)col * 27 * g.Nc + p0;
    T acc[V];
#pragma unroll
    for (int v = 0; v < V; v++) acc[v] = T(0);
#pragma unroll
    for (int q = 0; q < 27; q++) {
        if (q == 13) continue;
        T a[V];
        ld_stream_v(Ap + q * g.Nc, ps, a);
        long o = slot_off(g, q);
#pragma unroll
        for (int v = 0; v < V; v++) acc[v] = madd<true, T>(acc[v], a[v], ld_keep(x + xc[v] + o, pk));
    }
    T d[V], rv[V];
    ld_stream_v(Ap + 13 * g.Nc, ps, d);
    ld_stream_v(r + (long)col * g.Nc + p0, ps, rv);
#pragma unroll
    for (int v = 0; v < V; v++)
        if (ok[v]) st_keep(x + xc[v], mul_rn<T>(sub_rn<T>(rv[v], acc[v]), T(1) / d[v]), pk);
}

// The colour pass with the stencil prefetched before the launch dependency:
// launched as a programmatic dependent launch, a block may start while the
// previous kernel still runs.  Its 27 coefficients -- 90 % of the bytes,
// written only at set-up -- are loaded first; only then does it wait for
// the previous kernel and load the source and the neighbours' x, which that
// kernel may have written.  Same arithmetic as gs_value.
// Prefetch into L2 (cp.async.bulk.prefetch, the TMA's bulk prefetch) of the
// stencil runs and the source run of colour `col` for colour points [p0,
// p0 + L): 16-byte-aligned starts (slot planes on 256-byte boundaries, p0 a
// multiple of the block size), sizes rounded up to 16 bytes inside the
// plane's padding.  A cache hint: it changes no result.
template <class T>
__device__ __forceinline__ void prefetch_colour_l2(const LevelGeom& g, const T* A, const T* r, int col, long p0,
                                                   long L) {
    const unsigned bytes = (unsigned)((L * (long)sizeof(T) + 15) & ~15L);
    const T* Ap = A + (long)col * 27 * g.Nc + p0;
#pragma unroll 1
    for (int q = 0; q < 27; q++)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(Ap + q * g.Nc), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(r + (long)col * g.Nc + p0), "r"(bytes) : "memory");
}

// next >= 0: thread 0 of each block also prefetches colour `next`'s stencil
// and source for the block's points into L2 at the start, so that on levels
// whose colour fits in L2 the next pass reads them from there while this one
// runs.
template <class T, int BS>
__global__ void __launch_bounds__(BS) k_gs_colour_pf(LevelGeom g, T* x, const T* __restrict__ r,
                                                     const T* __restrict__ A, int col, int rev, int next) {
    long nc = (long)g.M2 * g.N2 * g.O2;
    unsigned b = rev ? gridDim.x - 1 - blockIdx.x : blockIdx.x;
    if (next >= 0 && threadIdx.x == 0) {
        long p0 = b * (long)BS;
        prefetch_colour_l2<T>(g, A, r, next, p0, nc - p0 < BS ? nc - p0 : BS);
    }
    long p = b * (long)BS + threadIdx.x;
    bool ok = p < nc;
    int i = 0, j = 0, k = 0;
    if (ok) {
        int i2, j2, k2;
        decode_colour(g, p, i2, j2, k2);
        i = 2 * i2 + (col & 1); j = 2 * j2 + ((col >> 1) & 1); k = 2 * k2 + (col >> 2);
        ok = i < g.m && j < g.n && k < g.o;
    }
    uint64_t ps = policy_evict_first(), pk = policy_evict_last();
    T a[27];
    if (ok) {
        const T* Ap = A + (long)col * 27 * g.Nc + p;
#pragma unroll
        for (int q = 0; q < 27; q++) a[q] = ld_stream(Ap + q * g.Nc, ps);
    }
    pdl_enter();
    if (!ok) return;
    long xc = g.xi(i, j, k);
    T rv = ld_stream(r + (long)col * g.Nc + p, ps);
    T acc = T(0);
#pragma unroll
    for (int q = 0; q < 27; q++) {
        if (q == 13) continue;
        acc = madd<true, T>(acc, a[q], ld_keep(x + xc + slot_off(g, q), pk));
    }
    st_keep(x + xc, mul_rn<T>(sub_rn<T>(rv, acc), T(1) / a[13]), pk);
}

// Hyperplane t = i + 2j + 4k of the lexicographic order.  Every neighbour of
// a 27-point box that precedes a point lexicographically lies on an earlier
// hyperplane (offsets (-1,0,0) -> -1; (+1,-1,0) -> -1; (d,d',-1) -> <= -1)
// and every later one on a later hyperplane, so sweeping hyperplanes in
// order, each fully in parallel, reproduces the reference's update order.
struct Plane {
    int kmin, kmax, jw;
};

__host__ __device__ inline Plane plane_range(const LevelGeom& g, int t) {
    Plane P;
    int hi = (g.m - 1) + 2 * (g.n - 1);
    int lo4 = t - hi;
    P.kmin = lo4 <= 0 ? 0 : (lo4 + 3) / 4;
    P.kmax = t / 4 < g.o - 1 ? t / 4 : g.o - 1;
    P.jw = (g.m + 1) / 2 + 1;
    return P;
}

__host__ __device__ inline int num_planes(const LevelGeom& g) {
    return (g.m - 1) + 2 * (g.n - 1) + 4 * (g.o - 1) + 1;
}

// Maps work item w of hyperplane t to a grid point; false if none.
__device__ __forceinline__ bool plane_point(const LevelGeom& g, const Plane& P, int t, int w,
                                            int& i, int& j, int& k) {
    k = P.kmin + w / P.jw;
    if (k > P.kmax) return false;
    int s = t - 4 * k;
    int jlo4 = s - (g.m - 1);
    int jmin = jlo4 <= 0 ? 0 : (jlo4 + 1) / 2;
    j = jmin + w % P.jw;
    if (j > g.n - 1 || 2 * j > s) return false;
    i = s - 2 * j;
    return i >= 0 && i < g.m;
}

// K2 (large levels): one hyperplane per launch.
template <class T>
__global__ void __launch_bounds__(kBlock) k_gs_plane(LevelGeom g, T* x, const T* __restrict__ r,
                                                     const T* __restrict__ A, int t, Plane P) {
    pdl_enter();
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!plane_point(g, P, t, w, i, j, k)) return;
    long xc = g.xi(i, j, k);
    int col = g.colour(i, j, k);
    long c = g.cidx(i, j, k);
    const T* Ap = A + (long)col * 27 * g.Nc + c;
    // x is read and written in this launch, but never the same address by
    // two threads of one hyperplane: plain loads, not the read-only path.
    T acc = T(0);
#pragma unroll
    for (int q = 0; q < 27; q++) {
        if (q == 13) continue;
        acc = madd<true, T>(acc, Ap[q * g.Nc], x[xc + slot_off(g, q)]);
    }
    T inv = T(1) / Ap[13 * g.Nc];
    x[xc] = mul_rn<T>(sub_rn<T>(r[(long)col * g.Nc + c], acc), inv);
}

// K2 (small levels): a whole level in one thread block, `sweeps` sweeps (each
// forward, plus backward if mode), hyperplanes separated by block barriers.
template <class T>
__global__ void __launch_bounds__(1024) k_gs_lex_block(LevelGeom g, T* x, const T* __restrict__ r,
                                                       const T* __restrict__ A, int sweeps, int mode) {
    pdl_enter();
    int np = num_planes(g);
    for (int s = 0; s < sweeps; s++) {
        for (int pass = 0; pass < (mode ? 2 : 1); pass++) {
            for (int tt = 0; tt < np; tt++) {
                int t = pass ? np - 1 - tt : tt;
                Plane P = plane_range(g, t);
                int nw = (P.kmax - P.kmin + 1) * P.jw;
                for (int w = threadIdx.x; w < nw; w += blockDim.x) {
                    int i, j, k;
                    if (!plane_point(g, P, t, w, i, j, k)) continue;
                    long xc = g.xi(i, j, k);
                    int col = g.colour(i, j, k);
                    long c = g.cidx(i, j, k);
                    const T* Ap = A + (long)col * 27 * g.Nc + c;
                    T acc = T(0);
#pragma unroll
                    for (int q = 0; q < 27; q++) {
                        if (q == 13) continue;
                        acc = madd<true, T>(acc, Ap[q * g.Nc], x[xc + slot_off(g, q)]);
                    }
                    T inv = T(1) / Ap[13 * g.Nc];
                    x[xc] = mul_rn<T>(sub_rn<T>(r[(long)col * g.Nc + c], acc), inv);
                }
                __syncthreads();
            }
        }
    }
}

// 8-colour sweep of a small level in one thread block (slab order as
// k_gs_colour's launches).
template <class T>
__global__ void __launch_bounds__(1024) k_gs_mc8_block(LevelGeom g, T* x, const T* __restrict__ r,
                                                       const T* __restrict__ A, int sweeps, int mode,
                                                       long long slab_budget) {
    pdl_enter();
    int S = slab_count(g, (int)sizeof(T), slab_budget);
    for (int s = 0; s < sweeps; s++) {
        for (int pass = 0; pass < (mode ? 2 : 1); pass++) {
            for (int ss = 0; ss < S; ss++) {
                int sl = pass ? S - 1 - ss : ss;
                long p0 = (long)slab_lo(g, sl, S) * g.M2 * g.N2, p1 = (long)slab_lo(g, sl + 1, S) * g.M2 * g.N2;
                for (int cc = 0; cc < 8; cc++) {
                    int col = colour_seq(pass ? 7 - cc : cc);
                    for (long p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
                        int i2, j2, k2;
                        decode_colour(g, p, i2, j2, k2);
                        int i = 2 * i2 + (col & 1), j = 2 * j2 + ((col >> 1) & 1), k = 2 * k2 + (col >> 2);
                        if (i >= g.m || j >= g.n || k >= g.o) continue;
                        long xc = g.xi(i, j, k);
                        const T* Ap = A + (long)col * 27 * g.Nc + p;
                        T acc = T(0);
#pragma unroll
                        for (int q = 0; q < 27; q++) {
                            if (q == 13) continue;
                            acc = madd<true, T>(acc, Ap[q * g.Nc], x[xc + slot_off(g, q)]);
                        }
                        x[xc] = mul_rn<T>(sub_rn<T>(r[(long)col * g.Nc + p], acc), T(1) / Ap[13 * g.Nc]);
                    }
                    __syncthreads();
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Block reduction of two doubles with a fixed tree (deterministic).
__device__ __forceinline__ void block_sum2(double& a, double& b, double* sh) {
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

// K5 / residual half of K3: res = r - A x over a whole level (all 27 slots in
// box order, region.cc:1833-1842), written colour-major to `out` (type TO),
// with per-block partial sums of res^2 and r^2 (region.cc:1475-1490,
// 1549-1558) when `partials` is non-null.  Grid: (blocks per colour, 8).
// Residual of colour point p of colour col: writes r - Ax to out (if
// non-null) and adds res^2 and r^2 to the accumulators.
template <class T, class TO>
__device__ __forceinline__ void residual_at(const LevelGeom& g, const T* __restrict__ x, const T* __restrict__ r,
                                            const T* __restrict__ A, TO* __restrict__ out, int col, long p,
                                            double& s_res, double& s_rhs) {
    long nc = (long)g.M2 * g.N2 * g.O2;
    if (p >= nc) return;
    int i2, j2, k2;
    decode_colour(g, p, i2, j2, k2);
    int i = 2 * i2 + (col & 1), j = 2 * j2 + ((col >> 1) & 1), k = 2 * k2 + (col >> 2);
    if (i >= g.m || j >= g.n || k >= g.o) return;
    uint64_t ps = policy_evict_first(), pk = policy_evict_last();
    long xc = g.xi(i, j, k);
    const T* Ap = A + (long)col * 27 * g.Nc + p;
    T acc = T(0);
#pragma unroll
    for (int q = 0; q < 27; q++)
        acc = madd<true, T>(acc, ld_stream(Ap + q * g.Nc, ps), ld_keep(x + xc + slot_off(g, q), pk));
    T rv = ld_stream(r + (long)col * g.Nc + p, ps);
    T res = sub_rn<T>(rv, acc);
    if (out) out[(long)col * g.Nc + p] = (TO)res;
    s_res = (double)res * (double)res;
    s_rhs = (double)rv * (double)rv;
}

// K5 / residual half of K3: res = r - A x over a whole level (all 27 slots in
// box order, region.cc:1833-1842), written colour-major to `out` (type TO),
// with per-block partial sums of res^2 and r^2 (region.cc:1475-1490,
// 1549-1558) when `partials` is non-null.  1D grid of 8 x (blocks per
// colour): block q is block q/8 of colour q%8, so the 8 colours of a region
// run side by side and share its x in L2 (colour by colour, a level whose x
// exceeds L2 re-reads it from HBM for every colour).  Block (colour c,
// block k) writes partial pair c * (blocks per colour) + k, the order the
// reduction sums them in.
__device__ __forceinline__ void colour_block(unsigned q, unsigned& col, unsigned& blk) {
    col = q & 7u;
    blk = q >> 3;
}

template <class T, class TO, bool EXACT>
__global__ void __launch_bounds__(kBlock) k_residual(LevelGeom g, const T* __restrict__ x,
                                                     const T* __restrict__ r, const T* __restrict__ A,
                                                     TO* __restrict__ out, double* __restrict__ partials) {
    pdl_enter();
    __shared__ double sh[64];
    unsigned col, blk;
    colour_block(blockIdx.x, col, blk);
    double s_res = 0, s_rhs = 0;
    residual_at<T, TO>(g, x, r, A, out, (int)col, blk * (long)blockDim.x + threadIdx.x, s_res, s_rhs);
    if (partials) {
        block_sum2(s_res, s_rhs, sh);
        if (threadIdx.x == 0) {
            long b = (long)col * (gridDim.x >> 3) + blk;
            partials[2 * b] = s_res;
            partials[2 * b + 1] = s_rhs;
        }
    }
}

// Sum of squared sources of a level (res^2 = r^2 when x = 0), optionally
// copying the source to `out` (the FP32 correction source of mixed
// precision).  Same grid and partials layout as k_residual.
template <class T, class TO>
__global__ void __launch_bounds__(kBlock) k_source(LevelGeom g, const T* __restrict__ r, TO* __restrict__ out,
                                                   double* __restrict__ partials) {
    pdl_enter();
    __shared__ double sh[64];
    unsigned ucol, blk;
    colour_block(blockIdx.x, ucol, blk);
    const int col = (int)ucol;
    long nc = (long)g.M2 * g.N2 * g.O2;
    long p = blk * (long)blockDim.x + threadIdx.x;
    double s = 0;
    if (p < nc) {
        T rv = r[(long)col * g.Nc + p];
        if (out) out[(long)col * g.Nc + p] = (TO)rv;
        s = (double)rv * (double)rv;
    }
    double s2 = s;
    block_sum2(s, s2, sh);
    if (threadIdx.x == 0) {
        long b = (long)col * (gridDim.x >> 3) + blk;
        partials[2 * b] = s;
        partials[2 * b + 1] = s2;
    }
}

// Sums nb partial pairs in a fixed order into out[0], out[1].
static __global__ void __launch_bounds__(1024) k_reduce_partials(const double* __restrict__ partials, long nb,
                                                          double* __restrict__ out) {
    pdl_enter();
    __shared__ double sh[64];
    double a = 0, b = 0;
    for (long q = threadIdx.x; q < nb; q += blockDim.x) { a += partials[2 * q]; b += partials[2 * q + 1]; }
    block_sum2(a, b, sh);
    if (threadIdx.x == 0) { out[0] = a; out[1] = b; }
}

// ---------------------------------------------------------------------------
// Restriction (region.cc:546-572, restrict_full/partial :818-912) as a gather
// per coarse point: contributions arrive in the reference's order -- cubes in
// scan order (z, then y, then x), fine points of a cube in x-fastest order --
// each 0.125*w*residual with w = product of per-axis transfer weights.  The
// reference's restrict_partial tests the x snap flag for the y axis of the
// (ti,tj+1,tk+1) point (region.cc:888-895); that is kept, see ysnap below.
// Also clears the coarse x (multigrid.cc:219).
template <class T, bool PRD, class Get>
__device__ __forceinline__ T restrict_sum(const LevelGeom& gf, int I, int J, int K, Get res) {
    // PRD: the instantiation for levels with periodic axes.
    const bool qx = PRD && px(gf), qy = PRD && py(gf), qz = PRD && pz(gf);
    int lx = cube_last(gf.m, qx), ly = cube_last(gf.n, qy), lz = cube_last(gf.o, qz);
    T acc = T(0);
    for (int cz = K - 1; cz <= K; cz++) {
        if (cz < cube_first(gf.o, qz) || cz > lz) continue;
        bool zsn = snapped(cz, gf.o, qz);
        for (int cy = J - 1; cy <= J; cy++) {
            if (cy < cube_first(gf.n, qy) || cy > ly) continue;
            for (int cx = I - 1; cx <= I; cx++) {
                if (cx < cube_first(gf.m, qx) || cx > lx) continue;
                bool xsn = snapped(cx, gf.m, qx);
                for (int dz = 0; dz < 2; dz++) {
                    if (dz && !has_upper(cz, gf.o, qz)) continue;
                    double wz = tweight(cz, dz, K, zsn);
                    if (wz == 0.0) continue;
                    for (int dy = 0; dy < 2; dy++) {
                        if (dy && !has_upper(cy, gf.n, qy)) continue;
                        for (int dx = 0; dx < 2; dx++) {
                            if (dx && !has_upper(cx, gf.m, qx)) continue;
                            bool ysn = (!dx && dy && dz) ? xsn : snapped(cy, gf.n, qy);
                            double w = tweight(cx, dx, I, xsn) * tweight(cy, dy, J, ysn) * wz;
                            if (w == 0.0) continue;
                            int fi = wrap(2 * cx + dx, gf.m, qx), fj = wrap(2 * cy + dy, gf.n, qy),
                                fk = wrap(2 * cz + dz, gf.o, qz);
                            T rd = (T)(0.125 * w) * res(fi, fj, fk);
                            acc = add_rn<T>(acc, rd);
                        }
                    }
                }
            }
        }
    }
    return acc;
}

template <class T, bool PRD = false>
__device__ __forceinline__ void restrict_at(const LevelGeom& gf, const LevelGeom& gc, const T* __restrict__ res,
                                            T* __restrict__ rc, T* __restrict__ xc, long q) {
    if (q >= gc.npts) return;
    int I, J, K;
    decode_nat(gc, q, I, J, K);
    rc[gc.ri(I, J, K)] = restrict_sum<T, PRD>(gf, I, J, K, [&](int i, int j, int k) { return res[gf.ri(i, j, k)]; });
    xc[gc.xi(I, J, K)] = T(0);
}

template <class T, bool PRD = false>
__global__ void __launch_bounds__(kBlock) k_restrict(LevelGeom gf, LevelGeom gc, const T* __restrict__ res,
                                                     T* __restrict__ rc, T* __restrict__ xc) {
    pdl_enter();
    restrict_at<T, PRD>(gf, gc, res, rc, xc, blockIdx.x * (long)blockDim.x + threadIdx.x);
}

// Value of fine role `role` (bit 0 x, 1 y, 2 z: upper point of the cube on
// that axis) of a cube with coarse corners v[0..7] (x fastest).  `full`: the
// cube is not the last one on any non-periodic axis; xs/ys/zs: its upper
// point on that axis snaps onto the next coarse point.
template <class T>
__device__ __forceinline__ T interp_val(int role, bool full, bool xs, bool ys, bool zs, const T (&v)[8]) {
    const T h = T(0.5), qq = T(0.25), e = T(0.125);
    T val;
    if (full) {
        switch (role) {
            case 0: val = v[0]; break;
            case 1: val = h * (v[0] + v[1]); break;
            case 2: val = h * (v[0] + v[2]); break;
            case 3: val = qq * (((v[0] + v[1]) + v[2]) + v[3]); break;
            case 4: val = h * (v[0] + v[4]); break;
            case 5: val = qq * ((v[0] + v[1]) + (v[4] + v[5])); break;
            case 6: val = qq * (((v[0] + v[2]) + v[4]) + v[6]); break;
            default: val = e * (((((((v[0] + v[1]) + v[2]) + v[3]) + (v[4] + v[5])) + v[6]) + v[7])); break;
        }
    } else {
        switch (role) {
            case 0: val = v[0]; break;
            case 1: val = xs ? v[1] : h * (v[0] + v[1]); break;
            case 2: val = ys ? v[2] : h * (v[0] + v[2]); break;
            case 4: val = zs ? v[4] : h * (v[0] + v[4]); break;
            case 5:
                val = zs ? (xs ? v[5] : h * (v[4] + v[5])) : (xs ? h * (v[1] + v[5]) : qq * (((v[0] + v[1]) + v[4]) + v[5]));
                break;
            case 6:
                val = zs ? (ys ? v[6] : h * (v[4] + v[6])) : (ys ? h * (v[2] + v[6]) : qq * (((v[0] + v[2]) + v[4]) + v[6]));
                break;
            default: {
                T t2 = ys ? (xs ? v[3] : h * (v[2] + v[3])) : (xs ? h * (v[1] + v[3]) : qq * (((v[0] + v[1]) + v[2]) + v[3]));
                if (role == 3) { val = t2; break; }
                T t3 = ys ? (xs ? v[7] : h * (v[6] + v[7])) : (xs ? h * (v[5] + v[7]) : qq * (((v[4] + v[5]) + v[6]) + v[7]));
                val = zs ? t3 : h * (t3 + t2);
            }
        }
    }
    return val;
}

// Interpolation with correction add (region.cc:576-593), one thread per
// 2x2x2 cube: each fine point belongs to exactly one cube (C = t>>1, role
// t&1 per axis) and gets the value interpolate_full (:752-772) or
// interpolate_partial (:779-810) would give it -- the two differ in how some
// sums associate; partial is used on the last cube of every row, row of
// every slice and slice.  The cube's 8 coarse corners are loaded once and its
// (up to) 8 fine points updated.  Cubes are enumerated like colour points
// (M2 x N2 x O2 of the fine level), so cube C covers fine 2C and 2C+1 (when
// < the axis size) on each axis -- every fine point exactly once.  Corners
// outside the coarse grid read the zero halo (on a periodic axis, the upper
// corner of the last cube is coarse 0's image there); the formulas never use
// them for fine points that exist.
template <class T>
__device__ __forceinline__ void interp_cube_at(const LevelGeom& gf, const LevelGeom& gc, T* __restrict__ xf,
                                               const T* __restrict__ xcv, long p) {
    if (p >= (long)gf.M2 * gf.N2 * gf.O2) return;
    int Cx, Cy, Cz;
    decode_colour(gf, p, Cx, Cy, Cz);
    long b = gc.xi(Cx, Cy, Cz);
    long sy = gc.mx, sz = gc.mx * gc.my;
    T v[8] = {xcv[b], xcv[b + 1], xcv[b + sy], xcv[b + sy + 1],
              xcv[b + sz], xcv[b + sz + 1], xcv[b + sz + sy], xcv[b + sz + sy + 1]};
    const bool qx = px(gf), qy = py(gf), qz = pz(gf);
    bool full = (even_prd(gf.m, qx) || Cx < cube_last(gf.m)) && (even_prd(gf.n, qy) || Cy < cube_last(gf.n)) &&
                (even_prd(gf.o, qz) || Cz < cube_last(gf.o));
    bool xs = snapped(Cx, gf.m, qx), ys = snapped(Cy, gf.n, qy), zs = snapped(Cz, gf.o, qz);
    int i0 = 2 * Cx, j0 = 2 * Cy, k0 = 2 * Cz;
    long f0 = gf.xi(i0, j0, k0);
    T old[8];
#pragma unroll
    for (int role = 0; role < 8; role++) {
        int dx = role & 1, dy = (role >> 1) & 1, dz = role >> 2;
        bool in = i0 + dx < gf.m && j0 + dy < gf.n && k0 + dz < gf.o;
        old[role] = in ? xf[f0 + dx + gf.mx * (dy + gf.my * dz)] : T(0);
    }
#pragma unroll
    for (int role = 0; role < 8; role++) {
        int dx = role & 1, dy = (role >> 1) & 1, dz = role >> 2;
        if (i0 + dx < gf.m && j0 + dy < gf.n && k0 + dz < gf.o)
            xf[f0 + dx + gf.mx * (dy + gf.my * dz)] = old[role] + interp_val<T>(role, full, xs, ys, zs, v);
    }
}

template <class T>
__global__ void __launch_bounds__(kBlock) k_interp_cube(LevelGeom gf, LevelGeom gc, T* __restrict__ xf,
                                                        const T* __restrict__ xcv) {
    pdl_enter();
    interp_cube_at<T>(gf, gc, xf, xcv, blockIdx.x * (long)blockDim.x + threadIdx.x);
}

// Restriction of a non-periodic level.  Coarse points interior on all three
// axes run restrict_sum's loops with the weights known at compile time (the
// same contributions in the same order, all 27 loads issued first); the
// others take restrict_sum itself.
template <class T, class Get>
__device__ __forceinline__ T restrict_inner_sum(int I, int J, int K, Get res);

template <class T, class Get>
__device__ __forceinline__ T restrict_fast_sum(const LevelGeom& gf, int I, int J, int K, Get res) {
    if (!(inner_axis(I, gf.m) && inner_axis(J, gf.n) && inner_axis(K, gf.o)))
        return restrict_sum<T, false>(gf, I, J, K, res);
    return restrict_inner_sum<T>(I, J, K, res);
}

// restrict_sum of a coarse point interior on every axis (inner_axis).
template <class T, class Get>
__device__ __forceinline__ T restrict_inner_sum(int I, int J, int K, Get res) {
    // Per axis: cube a (0: I-1, 1: I), role d -> fine offset 2a+d-2 from 2I,
    // weight 0 (not visited), 1/2, 1, 1/2.
    T rv[27];
#pragma unroll
    for (int oz = -1; oz <= 1; oz++)
#pragma unroll
        for (int oy = -1; oy <= 1; oy++)
#pragma unroll
            for (int ox = -1; ox <= 1; ox++) rv[(oz + 1) * 9 + (oy + 1) * 3 + (ox + 1)] = res(2 * I + ox, 2 * J + oy, 2 * K + oz);
    T acc = T(0);
#pragma unroll
    for (int az = 0; az < 2; az++)
#pragma unroll
        for (int ay = 0; ay < 2; ay++)
#pragma unroll
            for (int ax = 0; ax < 2; ax++)
#pragma unroll
                for (int dz = 0; dz < 2; dz++)
#pragma unroll
                    for (int dy = 0; dy < 2; dy++)
#pragma unroll
                        for (int dx = 0; dx < 2; dx++) {
                            int oz = 2 * az + dz - 2, oy = 2 * ay + dy - 2, ox = 2 * ax + dx - 2;
                            if (ox < -1 || oy < -1 || oz < -1) continue;
                            double wx = ox ? 0.5 : 1.0, wy = oy ? 0.5 : 1.0, wz = oz ? 0.5 : 1.0;
                            double w = wx * wy * wz;
                            T rd = (T)(0.125 * w) * rv[(oz + 1) * 9 + (oy + 1) * 3 + (ox + 1)];
                            acc = add_rn<T>(acc, rd);
                        }
    return acc;
}

template <class T>
__device__ __forceinline__ void restrict_fast_at(const LevelGeom& gf, const LevelGeom& gc, const T* __restrict__ res,
                                                 T* __restrict__ rc, T* __restrict__ xc, long q) {
    if (q >= gc.npts) return;
    int I, J, K;
    decode_nat(gc, q, I, J, K);
    rc[gc.ri(I, J, K)] = restrict_fast_sum<T>(gf, I, J, K, [&](int i, int j, int k) { return res[gf.ri(i, j, k)]; });
    xc[gc.xi(I, J, K)] = T(0);
}

// Restriction of a non-periodic level, interior coarse points first (see
// CoarseSplit): their sums run with the weights known at compile time, the
// shell's take restrict_sum.
template <class T>
__global__ void __launch_bounds__(kBlock) k_restrict_fast(LevelGeom gf, LevelGeom gc, CoarseSplit sp,
                                                          const T* __restrict__ res, T* __restrict__ rc,
                                                          T* __restrict__ xc) {
    pdl_enter();
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= gc.npts) return;
    auto get = [&](int i, int j, int k) { return res[gf.ri(i, j, k)]; };
    int I, J, K;
    if (split_point(gc, sp, q, I, J, K))
        rc[gc.ri(I, J, K)] = restrict_inner_sum<T>(I, J, K, get);
    else
        rc[gc.ri(I, J, K)] = restrict_sum<T, false>(gf, I, J, K, get);
    xc[gc.xi(I, J, K)] = T(0);
}

// Residual fused with the restriction of a non-periodic level
// (region::restriction, region.cc:546-572: the residual r - A x of every fine
// point, region.cc:1833-1842, gathered into the coarse r with the weights of
// restrict_full/partial, :818-912; the coarse x cleared, multigrid.cc:219),
// without a residual array in global memory.  A CTA owns a tile of TX x TY
// coarse points and walks up KC coarse planes.  For coarse plane K it
// computes the residuals of fine planes 2K and 2K+1 over the tile's fine
// footprint -- fine x in [2*I0-1, 2*(I0+TX)-1], y likewise -- into a ring
// of three fine planes in shared memory (plane 2K-1 is kept from the step
// before), two residuals per thread at a time, then every thread gathers its
// coarse point's contributions from the ring in the reference's order.  Each
// residual and each sum is the one k_residual and k_restrict_fast compute,
// so the coarse source is the same bit for bit.  The footprint's one-point
// rim is recomputed by the neighbouring tiles, which run at the same time, so
// its stencils are mostly re-read from L2.  The dynamic shared memory is
// 3 * (2TY+1) * (2TX+1) values of T.  Measured at 257^3 it is 2.4x (FP64) and
// 2.1x (FP32) slower than k_residual + k_restrict_fast (1.93 ms against 0.81
// ms at level 0): each thread computes about 70 residuals one after another
// as its CTA walks up the planes, where the residual pass has one per
// thread, and the saved round trip is only 16 of 248 bytes per fine point.
// It is an autotuned option, off by default.
template <int TX, int TY, int KC>
struct RrTile {
    static constexpr int tx = TX, ty = TY, kc = KC, threads = TX * TY;
    static constexpr int fx = 2 * TX + 1, fy = 2 * TY + 1;
    static constexpr int plane = fx * fy;
    template <class T> static constexpr size_t smem() { return 3 * (size_t)plane * sizeof(T); }
};
using RrSmall = RrTile<32, 8, 8>;

template <class T, class Tile>
__global__ void __launch_bounds__(Tile::threads) k_resrestrict(LevelGeom gf, LevelGeom gc, const T* __restrict__ x,
                                                               const T* __restrict__ r, const T* __restrict__ A,
                                                               T* __restrict__ rc, T* __restrict__ xc) {
    extern __shared__ __align__(16) unsigned char rr_raw[];
    T* ring = reinterpret_cast<T*>(rr_raw);
    constexpr int FX = Tile::fx, NP = Tile::plane;
    pdl_enter();
    const int I0 = blockIdx.x * Tile::tx, J0 = blockIdx.y * Tile::ty, K0 = blockIdx.z * Tile::kc;
    const int K1 = K0 + Tile::kc < gc.o ? K0 + Tile::kc : gc.o;
    const int fi0 = 2 * I0 - 1, fj0 = 2 * J0 - 1;
    const uint64_t ps = policy_evict_first(), pk = policy_evict_last();
    // Residual of footprint entry w of fine plane fk (false: outside the level).
    auto point = [&](int w, int fk, long& xcn, const T*& Ap, const T*& rp) -> bool {
        int fi = fi0 + w % FX, fj = fj0 + w / FX;
        if (fi < 0 || fi >= gf.m || fj < 0 || fj >= gf.n) return false;
        int col = gf.colour(fi, fj, fk);
        long c = gf.cidx(fi, fj, fk);
        xcn = gf.xi(fi, fj, fk);
        Ap = A + (long)col * 27 * gf.Nc + c;
        rp = r + (long)col * gf.Nc + c;
        return true;
    };
    auto fine_plane = [&](int fk) {
        if (fk < 0 || fk >= gf.o) return;
        T* dst = ring + (fk % 3) * NP;
        for (int w0 = threadIdx.x; w0 < NP; w0 += 2 * Tile::threads) {
            const int w1 = w0 + Tile::threads;
            long x0 = 0, x1 = 0;
            const T *A0 = A, *A1 = A, *r0 = r, *r1 = r;
            const bool v0 = point(w0, fk, x0, A0, r0);
            const bool v1 = w1 < NP && point(w1, fk, x1, A1, r1);
            if (!v0) x0 = x1, A0 = A1, r0 = r1;
            if (!v1) x1 = x0, A1 = A0, r1 = r0;
            if (!v0 && !v1) continue;
            T a0 = T(0), a1 = T(0);
#pragma unroll
            for (int q = 0; q < 27; q++) {
                const long o = slot_off(gf, q);
                a0 = madd<true, T>(a0, ld_stream(A0 + q * gf.Nc, ps), ld_keep(x + x0 + o, pk));
                a1 = madd<true, T>(a1, ld_stream(A1 + q * gf.Nc, ps), ld_keep(x + x1 + o, pk));
            }
            if (v0) dst[w0] = sub_rn<T>(ld_stream(r0, ps), a0);
            if (v1) dst[w1] = sub_rn<T>(ld_stream(r1, ps), a1);
        }
    };
    const int I = I0 + (int)threadIdx.x % Tile::tx, J = J0 + (int)threadIdx.x / Tile::tx;
    fine_plane(2 * K0 - 1);
    for (int K = K0; K < K1; K++) {
        fine_plane(2 * K);
        fine_plane(2 * K + 1);
        __syncthreads();
        if (I < gc.m && J < gc.n) {
            T v = restrict_fast_sum<T>(gf, I, J, K, [&](int i, int j, int k) {
                return ring[(k % 3) * NP + (j - fj0) * FX + (i - fi0)];
            });
            rc[gc.ri(I, J, K)] = v;
            xc[gc.xi(I, J, K)] = T(0);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Field movement between natural order (double, caller side) and the level
// layout.  Grid over natural points.
template <class T>
__global__ void __launch_bounds__(kBlock) k_nat_to_x(LevelGeom g, const double* __restrict__ src, T* __restrict__ x) {
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= g.npts) return;
    int i, j, k;
    decode_nat(g, q, i, j, k);
    x[g.xi(i, j, k)] = (T)src[q];
}
template <class T>
__global__ void __launch_bounds__(kBlock) k_x_to_nat(LevelGeom g, const T* __restrict__ x, double* __restrict__ dst) {
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= g.npts) return;
    int i, j, k;
    decode_nat(g, q, i, j, k);
    dst[q] = (double)x[g.xi(i, j, k)];
}
template <class T>
__global__ void __launch_bounds__(kBlock) k_nat_to_cm(LevelGeom g, const double* __restrict__ src, T* __restrict__ r) {
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= g.npts) return;
    int i, j, k;
    decode_nat(g, q, i, j, k);
    r[g.ri(i, j, k)] = (T)src[q];
}
template <class T>
__global__ void __launch_bounds__(kBlock) k_cm_to_nat(LevelGeom g, const T* __restrict__ r, double* __restrict__ dst) {
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= g.npts) return;
    int i, j, k;
    decode_nat(g, q, i, j, k);
    dst[q] = (double)r[g.ri(i, j, k)];
}

// Stencils of planes [k0,k1) from natural 27-slot doubles (src holds exactly
// those planes) into the colour-major layout; slots outside the point's box
// (if boxes are given) are stored as zero, since the reference never reads them.
template <class T>
__global__ void __launch_bounds__(kBlock) k_coef_to_cm(LevelGeom g, int k0, int k1, const double* __restrict__ src,
                                                       const int8_t* __restrict__ S, T* __restrict__ A) {
    long npl = (long)g.m * g.n * (k1 - k0);
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= npl * 27) return;
    long pt = q / 27;
    int s = (int)(q % 27);
    int i = (int)(pt % g.m); long t = pt / g.m; int j = (int)(t % g.n); int k = (int)(t / g.n) + k0;
    double v = src[q];
    if (S) {
        const int8_t* b = S + 6 * g.pi(i, j, k);
        int di = s % 3 - 1, dj = (s / 3) % 3 - 1, dk = s / 9 - 1;
        if (di < b[0] || di >= b[1] || dj < b[2] || dj >= b[3] || dk < b[4] || dk >= b[5]) v = 0.0;
    }
    A[g.ai(i, j, k, s)] = (T)v;
}

// Colour-major stencils of planes [k0,k1) back to natural 27-slot doubles
// (dst holds exactly those planes).
template <class T>
__global__ void __launch_bounds__(kBlock) k_cm_to_coef(LevelGeom g, int k0, int k1, const T* __restrict__ A,
                                                       double* __restrict__ dst) {
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= (long)g.m * g.n * (k1 - k0) * 27) return;
    long pt = q / 27;
    int s = (int)(q % 27);
    int i = (int)(pt % g.m); long t = pt / g.m; int j = (int)(t % g.n); int k = (int)(t / g.n) + k0;
    dst[q] = (double)A[g.ai(i, j, k, s)];
}

// Periodic images: every halo cell whose out-of-range coordinates are all
// on periodic axes takes the value of the interior point it wraps to (the
// reference's ghost exchange with itself, region.cc:1338-1469, on one
// process).  Halo cells enumerated face by face: z faces (whole (m+2)x(n+2)
// planes), then y faces (without z halo rows), then x faces.
template <class T>
__global__ void __launch_bounds__(kBlock) k_halo_wrap(LevelGeom g, T* __restrict__ x) {
    pdl_enter();
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long zf = 2L * g.mx * g.my, yf = 2L * g.mx * g.o, xf = 2L * g.n * g.o;
    int i, j, k;
    if (q < zf) {
        long t = q % (g.mx * g.my);
        i = (int)(t % g.mx) - 1; j = (int)(t / g.mx) - 1; k = q < g.mx * g.my ? -1 : g.o;
    } else if (q < zf + yf) {
        long t = q - zf, u = t % (g.mx * g.o);
        i = (int)(u % g.mx) - 1; k = (int)(u / g.mx); j = t < g.mx * g.o ? -1 : g.n;
    } else if (q < zf + yf + xf) {
        long t = q - zf - yf, u = t % ((long)g.n * g.o);
        j = (int)(u % g.n); k = (int)(u / g.n); i = t < (long)g.n * g.o ? -1 : g.m;
    } else {
        return;
    }
    bool ox = i < 0 || i >= g.m, oy = j < 0 || j >= g.n, oz = k < 0 || k >= g.o;
    if ((ox && !px(g)) || (oy && !py(g)) || (oz && !pz(g))) return;
    int wi = i < 0 ? g.m - 1 : (i >= g.m ? 0 : i);
    int wj = j < 0 ? g.n - 1 : (j >= g.n ? 0 : j);
    int wk = k < 0 ? g.o - 1 : (k >= g.o ? 0 : k);
    x[g.xi(i, j, k)] = x[g.xi(wi, wj, wk)];
}

__host__ __device__ inline long halo_cells(const LevelGeom& g) {
    return 2L * g.mx * g.my + 2L * g.mx * g.o + 2L * g.n * g.o;
}

// Interior of x set to zero (region::clear_x_field, region.cc:1679-1682).
template <class T>
__global__ void __launch_bounds__(kBlock) k_clear_x(LevelGeom g, T* __restrict__ x) {
    pdl_enter();
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= g.npts) return;
    int i, j, k;
    decode_nat(g, q, i, j, k);
    x[g.xi(i, j, k)] = T(0);
}

// region::setup_test (region.cc:1812-1826), one process.
template <class T>
__global__ void __launch_bounds__(kBlock) k_setup_test(LevelGeom g, T* x, T* r, int ca, int xfield) {
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= g.npts) return;
    int i, j, k;
    decode_nat(g, q, i, j, k);
    T v;
    switch (ca) {
        case 0: v = i; break;
        case 1: v = j; break;
        case 2: v = k; break;
        case 3: v = k + j + i; break;
        case 4: v = 0; break;
        case 5: v = (i == 7 && j == 7 && k == 7) ? 1 : 0; break;
        default: v = 1;
    }
    if (xfield) x[g.xi(i, j, k)] = v; else r[g.ri(i, j, k)] = v;
}

// out = A in (region::mul_A / Ax / unpadded_Ax, region.cc:1861-1912):
// natural-order input and output of one level, box-order accumulation.  On a
// periodic axis a neighbour outside the grid is its periodic image
// (unpadded_Ax's non_neg_mod, region.cc:1885-1887); on a non-periodic axis
// it carries a zero stencil entry and is skipped.
template <class T>
__global__ void __launch_bounds__(kBlock) k_apply(LevelGeom g, const T* __restrict__ A, const double* __restrict__ in,
                                                  double* __restrict__ out) {
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= g.npts) return;
    int i, j, k;
    decode_nat(g, q, i, j, k);
    double acc = 0.0;
    for (int s = 0; s < 27; s++) {
        int ii = wrap(i + s % 3 - 1, g.m, px(g)), jj = wrap(j + (s / 3) % 3 - 1, g.n, py(g)),
            kk = wrap(k + s / 9 - 1, g.o, pz(g));
        if (ii < 0 || jj < 0 || kk < 0 || ii >= g.m || jj >= g.n || kk >= g.o) continue;
        acc = __dadd_rn(acc, __dmul_rn((double)A[g.ai(i, j, k, s)], in[g.pi(ii, jj, kk)]));
    }
    out[q] = acc;
}

// Per-block partial sums for the PCG helpers, over the points of a level in
// natural order (grid over natural points):
//   what 0: sum x*r            (region::source_soln_dot, region.cc:1921-1931)
//   what 1: sum (ext - x)^2    (region::soln_diff, region.hh:226-236; ext natural)
//   what 2: max |r - A x|      (region::l0_error_all, region.cc:1492-1506)
// written to partials[2*block] (the pair layout of k_reduce_partials).
static __global__ void __launch_bounds__(kBlock) k_helper_partials(LevelGeom g, const double* __restrict__ x,
                                                                   const double* __restrict__ r,
                                                                   const double* __restrict__ A,
                                                                   const double* __restrict__ ext, int what,
                                                                   double* __restrict__ partials) {
    __shared__ double sh[64];
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    double v = 0.0;
    if (q < g.npts) {
        int i, j, k;
        decode_nat(g, q, i, j, k);
        long xc = g.xi(i, j, k);
        if (what == 0) {
            v = x[xc] * r[g.ri(i, j, k)];
        } else if (what == 1) {
            double d = ext[q] - x[xc];
            v = d * d;
        } else {
            long c = g.cidx(i, j, k);
            int col = g.colour(i, j, k);
            const double* Ap = A + (long)col * 27 * g.Nc + c;
            double acc = 0.0;
            for (int s = 0; s < 27; s++) acc = __dadd_rn(acc, __dmul_rn(Ap[s * g.Nc], x[xc + slot_off(g, s)]));
            v = fabs(__dsub_rn(r[(long)col * g.Nc + c], acc));
        }
    }
    if (what == 2) {
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
        int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
        if (l == 0) sh[w] = v;
        __syncthreads();
        if (w == 0) {
            v = l < nw ? sh[l] : 0.0;
            for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
        }
    } else {
        double u = 0;
        block_sum2(v, u, sh);
    }
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = v;
        partials[2 * blockIdx.x + 1] = 0.0;
    }
}

// Largest of nb partial values (partials[2*q]) into out[0].
static __global__ void __launch_bounds__(1024) k_reduce_max(const double* __restrict__ partials, long nb,
                                                            double* __restrict__ out) {
    __shared__ double sh[32];
    double v = 0.0;
    for (long q = threadIdx.x; q < nb; q += blockDim.x) v = fmax(v, partials[2 * q]);
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        v = l < nw ? sh[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
        if (l == 0) out[0] = v;
    }
}

// x = r on a level (region::copy_rhs_to_soln, region.cc:1935-1942).
template <class T>
__global__ void __launch_bounds__(kBlock) k_r_to_x(LevelGeom g, const T* __restrict__ r, T* __restrict__ x) {
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= g.npts) return;
    int i, j, k;
    decode_nat(g, q, i, j, k);
    x[g.xi(i, j, k)] = r[g.ri(i, j, k)];
}

// Elementwise casts used by mixed precision.
template <class TI, class TO>
__global__ void __launch_bounds__(kBlock) k_cast(const TI* __restrict__ in, TO* __restrict__ out, long n) {
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q < n) out[q] = (TO)in[q];
}

// x64 += x32 over the interior (FP64 update of iterative refinement).
static __global__ void __launch_bounds__(kBlock) k_add_correction(LevelGeom g, double* __restrict__ x64,
                                                           const float* __restrict__ e32) {
    pdl_enter();
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= g.npts) return;
    int i, j, k;
    decode_nat(g, q, i, j, k);
    long c = g.xi(i, j, k);
    x64[c] = x64[c] + (double)e32[c];
}

// The same update over the whole halo'd arrays, four entries per thread with
// 16-byte loads (both arrays 16-byte aligned, n = their length).  Halo
// entries are zero in both on non-periodic axes, and on periodic ones the
// images that the wrap after the update rewrites, so every interior value is
// k_add_correction's.
static __global__ void __launch_bounds__(kBlock) k_add_correction_flat(double* __restrict__ x64,
                                                                       const float* __restrict__ e32, long n) {
    pdl_enter();
    long q = (blockIdx.x * (long)blockDim.x + threadIdx.x) * 4;
    if (q + 4 <= n) {
        float4 e = *reinterpret_cast<const float4*>(e32 + q);
        double2 a = *reinterpret_cast<const double2*>(x64 + q);
        double2 b = *reinterpret_cast<const double2*>(x64 + q + 2);
        a.x = a.x + (double)e.x;
        a.y = a.y + (double)e.y;
        b.x = b.x + (double)e.z;
        b.y = b.y + (double)e.w;
        *reinterpret_cast<double2*>(x64 + q) = a;
        *reinterpret_cast<double2*>(x64 + q + 2) = b;
    } else {
        for (long i = q; i < n; i++) x64[i] = x64[i] + (double)e32[i];
    }
}

}  // namespace pgmg
