// The coarse tail of the V-cycle in one thread-block cluster.
//
// Levels below a few tens of thousands of points are latency-bound: one
// colour pass of a 17^3 level is a few microseconds of launch and drain for
// a megabyte of data.  This kernel runs every level from `first` down to the
// bottom and back up -- 8-colour sweeps, residual restriction, the bottom
// solve, interpolation -- inside a single cluster of CTAs on neighbouring SMs,
// separating dependent phases with hardware cluster barriers
// (barrier.cluster.arrive.release / wait.acquire) instead of kernel launches.
// The barriers are the hardware's; there are no software spin-waits.
//
// Data written by one phase and read by another CTA in a later phase (x, r,
// the residual scratch) is loaded with ld.global.cg (L2, never a stale L1
// line); read-only stencils and the coarse inverse go through the normal
// path.  When the kernel is launched with dynamic shared memory, the sweeps
// of every level whose copy fits run from shared memory instead
// (c_sweeps_shared): each CTA holds the level's x and its own points'
// stencils, and new values reach the CTAs that read them through distributed
// shared memory, ordered by the same release/acquire cluster barriers.  The
// arithmetic is the same as the grid kernels' (reference-order, no fused
// multiply-add), so the cluster path gives bit-identical results.
#pragma once
#include <cooperative_groups.h>

#include "layout.cuh"

namespace pgmg {

constexpr int kMaxLv = 16;

template <class T>
struct CoarsePlan {
    int first, nl;       // levels first..nl-1 run here
    int lu_ok;           // bottom: 1 = explicit-inverse solve, 0 = 24 sweeps
    long long slab_budget;  // slab order of the 8-colour sweeps (as the grid path)
    int v_down, v_up;       // sweeps on level l: v_down+l before, v_up+l-1 after (multigrid.cc:92,102)
    LevelGeom g[kMaxLv];
    const T* A[kMaxLv];
    T* x[kMaxLv];
    T* r[kMaxLv];
    T* res[kMaxLv];
    const double* Minv;
};

// Cluster barrier in its two halves: arrive (release: this thread's earlier
// writes become visible to the cluster) and wait (acquire).  Loads of data
// that no phase writes may be issued between the two, so that their latency
// overlaps the barrier.
__device__ __forceinline__ void cl_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cl_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_sync() {
    cl_arrive();
    cl_wait();
}

template <class T>
__device__ __forceinline__ void c_colour(const LevelGeom g, T* x, const T* r, const T* A, int col, long p0, long p1,
                                         int tid, int nth) {
    for (long p = p0 + tid; p < p1; p += nth) {
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
            acc = madd<true, T>(acc, __ldg(Ap + q * g.Nc), __ldcg(x + xc + slot_off(g, q)));
        }
        T inv = T(1) / __ldg(Ap + 13 * g.Nc);
        x[xc] = mul_rn<T>(sub_rn<T>(__ldcg(r + (long)col * g.Nc + p), acc), inv);
    }
}

// Sweeps of a level whose colours have at most one point per thread (the
// usual case: levels of <= 8 x 512 x cluster-size points), in one slab.
// Thread tid owns colour point tid of every colour -- the same (i2,j2,k2),
// decoded once -- and keeps the coefficients and source of its next colour
// in registers, fetched between the halves of the barrier before that
// colour's pass; only the neighbours' x values, which the previous pass may
// have written, are loaded after it.  Same arithmetic as c_colour.
template <class T>
__device__ __forceinline__ void c_sweeps_owned(const LevelGeom g, T* x, const T* r, const T* A, int sweeps,
                                               int mode, int tid) {
    long nc = (long)g.M2 * g.N2 * g.O2;
    bool have = tid < nc;
    int i0 = 0, j0 = 0, k0 = 0;
    if (have) {
        int i2, j2, k2;
        decode_colour(g, tid, i2, j2, k2);
        i0 = 2 * i2; j0 = 2 * j2; k0 = 2 * k2;
    }
    const long xc0 = g.xi(i0, j0, k0), sy = g.mx, sz = g.mx * g.my;
    const int per = mode ? 16 : 8, total = sweeps * per;
    T a[27];
    T rv = T(0), ainv = T(1);
    auto colour_at = [&](int st) {
        int cc = st % per;
        return colour_seq(cc < 8 ? cc : 15 - cc);
    };
    auto valid = [&](int col) {
        return have && i0 + (col & 1) < g.m && j0 + ((col >> 1) & 1) < g.n && k0 + (col >> 2) < g.o;
    };
    auto fetch = [&](int col) {
        if (!valid(col)) return;
        const T* Ap = A + (long)col * 27 * g.Nc + tid;
#pragma unroll
        for (int q = 0; q < 27; q++) a[q] = __ldg(Ap + q * g.Nc);
        rv = __ldcg(r + (long)col * g.Nc + tid);
        ainv = T(1) / a[13];  // off the pass's critical path
    };
    if (total > 0) fetch(colour_at(0));
    for (int st = 0; st < total; st++) {
        int col = colour_at(st);
        if (valid(col)) {
            long xc = xc0 + (col & 1) + ((col >> 1) & 1) * sy + (col >> 2) * sz;
            T acc = T(0);
#pragma unroll
            for (int q = 0; q < 27; q++) {
                if (q == 13) continue;
                acc = madd<true, T>(acc, a[q], __ldcg(x + xc + slot_off(g, q)));
            }
            x[xc] = mul_rn<T>(sub_rn<T>(rv, acc), ainv);
        }
        cl_arrive();
        if (st + 1 < total) fetch(colour_at(st + 1));
        cl_wait();
    }
}

// Distributed shared memory helpers: a CTA's shared-window address, the same
// offset in the shared memory of CTA `rank` of the cluster, and a store there.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint32_t cl_map(uint32_t a, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}
__device__ __forceinline__ void st_cl(uint32_t a, double v) {
    asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
__device__ __forceinline__ void st_cl(uint32_t a, float v) {
    asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}
__device__ __forceinline__ unsigned dyn_smem_bytes() {
    unsigned r;
    asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(r));
    return r;
}

// Shared-memory copy of a level for c_sweeps_shared: the halo'd x array in
// its global (natural) layout, then the staged stencils.
struct ShCopy {
    long nc;      // colour points per colour
    long chunk;   // colour points owned per CTA
    long xelems;  // elements of the x copy (the halo'd array, rounded up to even)
    __host__ __device__ long bytes(int tsize) const { return (xelems + 8 * 28 * chunk) * tsize; }
};
__host__ __device__ inline ShCopy shared_copy(const LevelGeom& g, int csize) {
    ShCopy c;
    c.nc = (long)g.M2 * g.N2 * g.O2;
    c.chunk = (c.nc + csize - 1) / csize;
    c.xelems = (g.xsize() + 1) & ~1L;
    return c;
}

// c_sweeps_owned with the level held in shared memory.  Every CTA of the
// cluster keeps a copy of the halo'd x array (copied in from global memory
// at the start) and the coefficients, source and diagonal reciprocal of the
// points it owns (as[colour][28][chunk]: slots 0..26 the stencil with slot 13
// holding 1/diagonal, slot 27 the source).  Colour points are owned in
// contiguous chunks, one per CTA.  A pass reads the neighbours from the
// CTA's own copy (a neighbour's offset is the same for every colour, so a
// read is one add and one load) and writes each new value into the copies of
// the CTAs that own a point within reach of it (its neighbours lie within
// +-(M2*N2 + M2 + 1) colour points) with st.shared::cluster stores, ordered
// by the same cluster barriers: no pass waits for L2.  A CTA's copy is
// current for the points its own points read.  At the end each owner writes
// its points back to global memory.  Same arithmetic as c_sweeps_owned.
template <class T>
__device__ __noinline__ void c_sweeps_shared(const LevelGeom g, T* x, const T* r, const T* A, int sweeps,
                                             int mode, T* sm, int rank, int csize) {
    const ShCopy cp = shared_copy(g, csize);
    const int nc = (int)cp.nc, chunk = (int)cp.chunk;
    const int p = rank * chunk + (int)threadIdx.x;
    const bool have = (int)threadIdx.x < chunk && p < nc;
    int i2 = 0, j2 = 0, k2 = 0;
    if (have) decode_colour(g, p, i2, j2, k2);
    // Shared-memory indexes fit in 32 bits (the copies are at most kCoarseXsMax bytes).
    const int mxi = (int)g.mx, szi = (int)(g.mx * g.my);
    const int xc0 = (int)g.xi(2 * i2, 2 * j2, 2 * k2);
    T* as = sm + cp.xelems;
    const int xn = (int)g.xsize();
    for (int e = threadIdx.x; e < xn; e += blockDim.x) sm[e] = __ldcg(x + e);
    auto valid = [&](int col) {
        return have && 2 * i2 + (col & 1) < g.m && 2 * j2 + ((col >> 1) & 1) < g.n && 2 * k2 + (col >> 2) < g.o;
    };
    auto at = [&](int col) { return xc0 + (col & 1) + ((col >> 1) & 1) * mxi + (col >> 2) * szi; };
    for (int col = 0; col < 8; col++) {
        // Thread t stages its own points and reads them back itself.
        if (!valid(col)) continue;
        const T* Ap = A + (long)col * 27 * g.Nc + p;
        T* sp = as + col * 28 * chunk + threadIdx.x;
#pragma unroll
        for (int q = 0; q < 27; q++) sp[q * chunk] = q == 13 ? T(1) / __ldg(Ap + 13 * g.Nc) : __ldg(Ap + q * g.Nc);
        sp[27 * chunk] = __ldcg(r + (long)col * g.Nc + p);
    }
    // CTAs whose points read this CTA's points.
    const int span = g.M2 * g.N2 + g.M2 + 1;
    const int plo = rank * chunk - span, phi = (rank + 1) * chunk - 1 + span;
    const int dlo = plo < 0 ? 0 : plo / chunk;
    const int dhi = phi / chunk < csize - 1 ? phi / chunk : csize - 1;
    const uint32_t base = smem_u32(sm);
    const int per = mode ? 16 : 8, total = sweeps * per;
    // Every copy is complete before any CTA writes into another's.
    cluster_sync();
    for (int st = 0; st < total; st++) {
        int cc = st % per;
        int col = colour_seq(cc < 8 ? cc : 15 - cc);
        if (valid(col)) {
            const T* sp = as + col * 28 * chunk + threadIdx.x;
            const int xc = at(col);
            const T* xp = sm + xc;
            T acc = T(0);
#pragma unroll
            for (int q = 0; q < 27; q++) {
                if (q == 13) continue;
                acc = madd<true, T>(acc, sp[q * chunk], xp[(q % 3 - 1) + mxi * ((q / 3) % 3 - 1) + szi * (q / 9 - 1)]);
            }
            T v = mul_rn<T>(sub_rn<T>(sp[27 * chunk], acc), sp[13 * chunk]);
            uint32_t off = base + (uint32_t)xc * (uint32_t)sizeof(T);
            for (int d = dlo; d <= dhi; d++) st_cl(cl_map(off, (uint32_t)d), v);
        }
        cluster_sync();
    }
    for (int col = 0; col < 8; col++)
        if (valid(col)) x[at(col)] = sm[at(col)];
    cluster_sync();
}

// Halo'd z planes [lo, hi] of a level that CTA `rank` of a `csize`-CTA
// cluster needs when it owns colour points [rank*chunk, (rank+1)*chunk) of
// every colour (c_sweeps_shared's ownership): the fine planes of its points
// and one more on each side.  hi < lo when it owns none.
__host__ __device__ inline void win_planes(const LevelGeom& g, int rank, int csize, int& lo, int& hi) {
    const long nc = (long)g.M2 * g.N2 * g.O2, chunk = (nc + csize - 1) / csize, pl = (long)g.M2 * g.N2;
    const long p0 = (long)rank * chunk, p1 = ((long)(rank + 1) * chunk < nc ? (long)(rank + 1) * chunk : nc) - 1;
    if (p0 >= nc) {
        lo = 0;
        hi = -1;
        return;
    }
    const int k2lo = (int)(p0 / pl), k2hi = (int)(p1 / pl);
    lo = 2 * k2lo;                                      // fine plane 2*k2lo - 1, halo'd
    hi = 2 * k2hi + 3 < g.o + 1 ? 2 * k2hi + 3 : g.o + 1;  // fine plane 2*k2hi + 2, halo'd
}
// Bytes of the largest window of a level over the CTAs of the cluster.
__host__ __device__ inline long window_bytes(const LevelGeom& g, int csize, int tsize) {
    long w = 0;
    for (int d = 0; d < csize; d++) {
        int lo, hi;
        win_planes(g, d, csize, lo, hi);
        long b = (long)(hi - lo + 1) * g.mx * g.my * tsize;
        if (b > w) w = b;
    }
    return w;
}

// The sweeps of a level whose full shared copy (c_sweeps_shared) does not
// fit, with x from shared memory all the same: each CTA holds only the window
// of halo'd z planes its own points and their neighbours lie in (win_planes;
// points owned as in c_sweeps_shared), loaded from global memory at the
// start.  A new value goes with st.shared::cluster stores into the window of
// every CTA that holds its plane, ordered by the release/acquire cluster
// barrier of the pass.  The stencil, source and diagonal reciprocal of a
// thread's next colour are fetched from L2 into registers between the halves
// of that barrier, as in c_sweeps_owned.  At the end each owner writes its
// points back.  Same arithmetic as c_sweeps_owned.
template <class T>
__device__ __noinline__ void c_sweeps_window(const LevelGeom g, T* x, const T* r, const T* A, int sweeps, int mode,
                                             T* sm, int rank, int csize) {
    const long nc = (long)g.M2 * g.N2 * g.O2;
    const int chunk = (int)((nc + csize - 1) / csize);
    const int p = rank * chunk + (int)threadIdx.x;
    const bool have = (int)threadIdx.x < chunk && p < nc;
    int i2 = 0, j2 = 0, k2 = 0;
    if (have) decode_colour(g, p, i2, j2, k2);
    // Shared-memory indexes fit in 32 bits (a window is at most kCoarseXsMax bytes).
    const int mxi = (int)g.mx, szi = (int)(g.mx * g.my);
    int lo, hi;
    win_planes(g, rank, csize, lo, hi);
    const int wbase = lo * szi;
    for (int e = threadIdx.x; e < (hi - lo + 1) * szi; e += blockDim.x) sm[e] = __ldcg(x + wbase + e);
    const int xc0 = (int)g.xi(2 * i2, 2 * j2, 2 * k2);
    auto valid = [&](int col) {
        return have && 2 * i2 + (col & 1) < g.m && 2 * j2 + ((col >> 1) & 1) < g.n && 2 * k2 + (col >> 2) < g.o;
    };
    auto at = [&](int col) { return xc0 + (col & 1) + ((col >> 1) & 1) * mxi + (col >> 2) * szi; };
    const int per = mode ? 16 : 8, total = sweeps * per;
    auto colour_at = [&](int st) {
        int cc = st % per;
        return colour_seq(cc < 8 ? cc : 15 - cc);
    };
    T a[27];
    T rv = T(0), ainv = T(1);
    auto fetch = [&](int col) {
        if (!valid(col)) return;
        const T* Ap = A + (long)col * 27 * g.Nc + p;
#pragma unroll
        for (int q = 0; q < 27; q++) a[q] = __ldg(Ap + q * g.Nc);
        rv = __ldcg(r + (long)col * g.Nc + p);
        ainv = T(1) / a[13];
    };
    const uint32_t base = smem_u32(sm);
    if (total > 0) fetch(colour_at(0));
    // Every window is loaded before any CTA writes into another's.
    cluster_sync();
    for (int st = 0; st < total; st++) {
        int col = colour_at(st);
        if (valid(col)) {
            const int gi = at(col);
            const T* xp = sm + (gi - wbase);
            T acc = T(0);
#pragma unroll
            for (int q = 0; q < 27; q++) {
                if (q == 13) continue;
                acc = madd<true, T>(acc, a[q], xp[(q % 3 - 1) + mxi * ((q / 3) % 3 - 1) + szi * (q / 9 - 1)]);
            }
            const T v = mul_rn<T>(sub_rn<T>(rv, acc), ainv);
            const int hz = gi / szi;
            for (int d = 0; d < csize; d++) {
                int dl, dh;
                win_planes(g, d, csize, dl, dh);
                if (hz < dl || hz > dh) continue;
                st_cl(cl_map(base + (uint32_t)(gi - dl * szi) * (uint32_t)sizeof(T), (uint32_t)d), v);
            }
        }
        cl_arrive();
        if (st + 1 < total) fetch(colour_at(st + 1));
        cl_wait();
    }
    for (int col = 0; col < 8; col++)
        if (valid(col)) x[at(col)] = sm[at(col) - wbase];
    cluster_sync();
}

template <class T>
__device__ __forceinline__ void c_sweeps(const LevelGeom g, T* x, const T* r, const T* A, int sweeps, int mode,
                                         long long budget, int tid, int nth, T* xs, int rank, int csize) {
    int S = slab_count(g, (int)sizeof(T), budget);
    if (S == 1 && (long)g.M2 * g.N2 * g.O2 <= nth) {
        if (xs && shared_copy(g, csize).bytes((int)sizeof(T)) <= (long)dyn_smem_bytes())
            c_sweeps_shared<T>(g, x, r, A, sweeps, mode, xs, rank, csize);
        else if (xs && (long)((g.M2 * g.N2 * g.O2 + csize - 1) / csize) <= (long)blockDim.x &&
                 window_bytes(g, csize, (int)sizeof(T)) <= (long)dyn_smem_bytes())
            c_sweeps_window<T>(g, x, r, A, sweeps, mode, xs, rank, csize);
        else
            c_sweeps_owned<T>(g, x, r, A, sweeps, mode, tid);
        return;
    }
    for (int s = 0; s < sweeps; s++)
        for (int pass = 0; pass < (mode ? 2 : 1); pass++)
            for (int ss = 0; ss < S; ss++) {
                int sl = pass ? S - 1 - ss : ss;
                long p0 = (long)slab_lo(g, sl, S) * g.M2 * g.N2, p1 = (long)slab_lo(g, sl + 1, S) * g.M2 * g.N2;
                for (int cc = 0; cc < 8; cc++) {
                    c_colour<T>(g, x, r, A, colour_seq(pass ? 7 - cc : cc), p0, p1, tid, nth);
                    cluster_sync();
                }
            }
}

template <class T>
__device__ __forceinline__ void c_residual(const LevelGeom g, const T* x, const T* r, const T* A, T* res, int tid,
                                           int nth) {
    long nc = (long)g.M2 * g.N2 * g.O2;
    for (long pp = tid; pp < 8 * nc; pp += nth) {
        int col = (int)(pp / nc);
        long p = pp % nc;
        int i2, j2, k2;
        decode_colour(g, p, i2, j2, k2);
        int i = 2 * i2 + (col & 1), j = 2 * j2 + ((col >> 1) & 1), k = 2 * k2 + (col >> 2);
        if (i >= g.m || j >= g.n || k >= g.o) continue;
        long xc = g.xi(i, j, k);
        const T* Ap = A + (long)col * 27 * g.Nc + p;
        T acc = T(0);
#pragma unroll
        for (int q = 0; q < 27; q++) acc = madd<true, T>(acc, __ldg(Ap + q * g.Nc), __ldcg(x + xc + slot_off(g, q)));
        res[(long)col * g.Nc + p] = sub_rn<T>(__ldcg(r + (long)col * g.Nc + p), acc);
    }
}

// Same accumulation order as k_restrict (reference restriction order).
template <class T>
__device__ __forceinline__ void c_restrict(const LevelGeom gf, const LevelGeom gc, const T* res, T* rc, T* xc,
                                           int tid, int nth) {
    int lx = cube_last(gf.m), ly = cube_last(gf.n), lz = cube_last(gf.o);
    for (long q = tid; q < gc.npts; q += nth) {
        int I, J, K;
        decode_nat(gc, q, I, J, K);
        T acc = T(0);
        for (int cz = K - 1; cz <= K; cz++) {
            if (cz < 0 || cz > lz) continue;
            bool zsn = snapped(cz, gf.o);
            for (int cy = J - 1; cy <= J; cy++) {
                if (cy < 0 || cy > ly) continue;
                for (int cx = I - 1; cx <= I; cx++) {
                    if (cx < 0 || cx > lx) continue;
                    bool xsn = snapped(cx, gf.m);
                    for (int dz = 0; dz < 2; dz++) {
                        if (dz && !has_upper(cz, gf.o)) continue;
                        double wz = tweight(cz, dz, K, zsn);
                        if (wz == 0.0) continue;
                        for (int dy = 0; dy < 2; dy++) {
                            if (dy && !has_upper(cy, gf.n)) continue;
                            for (int dx = 0; dx < 2; dx++) {
                                if (dx && !has_upper(cx, gf.m)) continue;
                                bool ysn = (!dx && dy && dz) ? xsn : snapped(cy, gf.n);
                                double w = tweight(cx, dx, I, xsn) * tweight(cy, dy, J, ysn) * wz;
                                if (w == 0.0) continue;
                                T rd = (T)(0.125 * w) * __ldcg(res + gf.ri(2 * cx + dx, 2 * cy + dy, 2 * cz + dz));
                                acc = add_rn<T>(acc, rd);
                            }
                        }
                    }
                }
            }
        }
        rc[gc.ri(I, J, K)] = acc;
        xc[gc.xi(I, J, K)] = T(0);
    }
}

// Same values as k_interp_cube (interp_val's formulas, inlined).
template <class T>
__device__ __forceinline__ void c_interp(const LevelGeom gf, const LevelGeom gc, T* xf, const T* xcv, int tid,
                                         int nth) {
    for (long q = tid; q < gf.npts; q += nth) {
        int i, j, k;
        decode_nat(gf, q, i, j, k);
        int Cx = i >> 1, Cy = j >> 1, Cz = k >> 1, dx = i & 1, dy = j & 1, dz = k & 1;
        long b = gc.xi(Cx, Cy, Cz);
        long sy = gc.mx, sz = gc.mx * gc.my;
        T v0 = __ldcg(xcv + b), v1 = __ldcg(xcv + b + 1), v2 = __ldcg(xcv + b + sy), v3 = __ldcg(xcv + b + sy + 1);
        T v4 = __ldcg(xcv + b + sz), v5 = __ldcg(xcv + b + sz + 1), v6 = __ldcg(xcv + b + sz + sy),
          v7 = __ldcg(xcv + b + sz + sy + 1);
        const T h = T(0.5), qq = T(0.25), e = T(0.125);
        int role = dx | (dy << 1) | (dz << 2);
        T val;
        bool full = Cx < cube_last(gf.m) && Cy < cube_last(gf.n) && Cz < cube_last(gf.o);
        if (full) {
            switch (role) {
                case 0: val = v0; break;
                case 1: val = h * (v0 + v1); break;
                case 2: val = h * (v0 + v2); break;
                case 3: val = qq * (((v0 + v1) + v2) + v3); break;
                case 4: val = h * (v0 + v4); break;
                case 5: val = qq * ((v0 + v1) + (v4 + v5)); break;
                case 6: val = qq * (((v0 + v2) + v4) + v6); break;
                default: val = e * (((((((v0 + v1) + v2) + v3) + (v4 + v5)) + v6) + v7)); break;
            }
        } else {
            bool xs = snapped(Cx, gf.m), ys = snapped(Cy, gf.n), zs = snapped(Cz, gf.o);
            switch (role) {
                case 0: val = v0; break;
                case 1: val = xs ? v1 : h * (v0 + v1); break;
                case 2: val = ys ? v2 : h * (v0 + v2); break;
                case 4: val = zs ? v4 : h * (v0 + v4); break;
                case 5: val = zs ? (xs ? v5 : h * (v4 + v5)) : (xs ? h * (v1 + v5) : qq * (((v0 + v1) + v4) + v5)); break;
                case 6: val = zs ? (ys ? v6 : h * (v4 + v6)) : (ys ? h * (v2 + v6) : qq * (((v0 + v2) + v4) + v6)); break;
                default: {
                    T t2 = ys ? (xs ? v3 : h * (v2 + v3)) : (xs ? h * (v1 + v3) : qq * (((v0 + v1) + v2) + v3));
                    if (role == 3) { val = t2; break; }
                    T t3 = ys ? (xs ? v7 : h * (v6 + v7)) : (xs ? h * (v5 + v7) : qq * (((v4 + v5) + v6) + v7));
                    val = zs ? t3 : h * (t3 + t2);
                }
            }
        }
        long xf_i = gf.xi(i, j, k);
        xf[xf_i] = __ldcg(xf + xf_i) + val;
    }
}

// x = Minv r on the bottom level, one warp per row (same reduction as
// k_lu_apply).  Levels of up to kLuShared points first gather the source into
// every CTA's shared memory in natural order, so the row products read it
// there instead of decoding and loading each entry from L2.
constexpr int kLuShared = 1024;

template <class T>
__device__ __forceinline__ void c_lu_apply(const LevelGeom g, const double* Minv, const T* r, T* x, int tid, int nth,
                                           double* sh) {
    int n = (int)g.npts;
    int lane = tid & 31;
    if (n <= kLuShared) {
        for (int c = threadIdx.x; c < n; c += blockDim.x) {
            int i = c % g.m, t = c / g.m, j = t % g.n, k = t / g.n;
            sh[c] = (double)__ldcg(r + g.ri(i, j, k));
        }
        __syncthreads();
    }
    for (int row = tid >> 5; row < n; row += nth >> 5) {
        double s = 0.0;
        if (n <= kLuShared) {
            const double* Mr = Minv + (long)row * n;
            for (int c = lane; c < n; c += 32) s = fma(__ldg(Mr + c), sh[c], s);
        } else {
            for (int c = lane; c < n; c += 32) {
                int i = c % g.m, t = c / g.m, j = t % g.n, k = t / g.n;
                s = fma(Minv[(long)row * n + c], (double)__ldcg(r + g.ri(i, j, k)), s);
            }
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) {
            int i = row % g.m, t = row / g.m, j = t % g.n, k = t / g.n;
            x[g.xi(i, j, k)] = (T)s;
        }
    }
}

// The V-cycle from level `first` (its source already restricted) to the
// bottom and back, 8-colour smoothing: v_down+l pre- and v_up+l-1 post-sweeps
// on level l (multigrid.cc:88-106).  One cluster per problem: cluster c runs
// plans[slot_of_cluster[c]] (plans[c] if the map is null) and returns at once
// if that problem's active flag is 0.  blockDim.x must be a multiple of 32.
template <class T>
__global__ void __launch_bounds__(512) k_coarse_cycle(const CoarsePlan<T>* __restrict__ plans,
                                                      const int* __restrict__ slot_of_cluster,
                                                      const int* __restrict__ active, int mode) {
    pdl_enter();
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    int csize = (int)cl.num_blocks();
    int cid = blockIdx.x / csize;
    int slot = slot_of_cluster ? slot_of_cluster[cid] : cid;
    // The flag is uniform across the cluster (written by an earlier kernel),
    // so either every CTA of the cluster returns here or none does.
    if (active && !active[slot]) return;
    const CoarsePlan<T>& P = plans[slot];
    int nth = csize * blockDim.x;
    int rank = (int)cl.block_rank();
    int tid = rank * blockDim.x + threadIdx.x;
    int nl = P.nl;
    // Shared copy of a level's x for the sweeps (when launched with dynamic
    // shared memory; every CTA of the cluster has the same amount).
    extern __shared__ __align__(16) unsigned char c_dyn[];
    T* xs = dyn_smem_bytes() > 0 ? reinterpret_cast<T*>(c_dyn) : nullptr;
    for (int l = P.first; l < nl - 1; l++) {
        c_sweeps<T>(P.g[l], P.x[l], P.r[l], P.A[l], P.v_down + l, mode, P.slab_budget, tid, nth, xs, rank, csize);
        c_residual<T>(P.g[l], P.x[l], P.r[l], P.A[l], P.res[l], tid, nth);
        cluster_sync();
        c_restrict<T>(P.g[l], P.g[l + 1], P.res[l], P.r[l + 1], P.x[l + 1], tid, nth);
        cluster_sync();
    }
    int lb = nl - 1;
    if (P.lu_ok) {
        __shared__ double sh_src[kLuShared];
        c_lu_apply<T>(P.g[lb], P.Minv, P.r[lb], P.x[lb], tid, nth, sh_src);
        cluster_sync();
    } else {
        c_sweeps<T>(P.g[lb], P.x[lb], P.r[lb], P.A[lb], 24, 0, P.slab_budget, tid, nth, xs, rank, csize);
    }
    for (int l = lb; l > P.first; l--) {
        c_interp<T>(P.g[l - 1], P.g[l], P.x[l - 1], P.x[l], tid, nth);
        cluster_sync();
        c_sweeps<T>(P.g[l - 1], P.x[l - 1], P.r[l - 1], P.A[l - 1], P.v_up + l - 1, mode, P.slab_budget, tid, nth, xs,
                    rank, csize);
    }
}

}  // namespace pgmg
