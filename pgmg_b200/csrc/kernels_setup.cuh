// Set-up kernels: Galerkin coarse operators (RAT) and their boxes, and the
// coarsest-level dense LU.  FP64 throughout.
#pragma once
#include <cooperative_groups.h>

#include "layout.cuh"

namespace pgmg {

// Per-axis list of the fine points (cube C, role d, weight w, A_mul factor f)
// that transfer to coarse index I, in scan order (cube I-1 first, lower role
// first).  At most 3 entries.
struct AxisList {
    int n;
    int C[3], d[3];
    double w[3], f[3];
};

__device__ inline AxisList axis_list(int I, int ma, bool p) {
    AxisList L;
    L.n = 0;
    int last = cube_last(ma, p);
    for (int C = I - 1; C <= I; C++) {
        if (C < cube_first(ma, p) || C > last) continue;
        bool sn = snapped(C, ma, p);
        for (int d = 0; d < 2; d++) {
            if (d && !has_upper(C, ma, p)) continue;
            double w = tweight(C, d, I, sn);
            if (w == 0.0) continue;
            L.C[L.n] = C; L.d[L.n] = d; L.w[L.n] = w;
            L.f[L.n] = (d && !sn) ? 0.5 : 1.0;
            L.n++;
        }
    }
    return L;
}

// fill_rat_bounds (region.cc:598-623; rat_bound_full/partial :916-1003;
// b_red :1105-1110; b_ex :1276-1283): coarse box = [0,1)^3 extended by the
// grid_map'ed global box of every fine point that transfers to the coarse
// point.  One thread per coarse point; boxes as int8[6] natural order.
static __global__ void __launch_bounds__(256) k_rat_bounds(LevelGeom gf, LevelGeom gc, const int8_t* __restrict__ Sf,
                                                    int8_t* __restrict__ Sc) {
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= gc.npts) return;
    int I, J, K;
    decode_nat(gc, q, I, J, K);
    int s[6] = {0, 1, 0, 1, 0, 1};
    const bool qx = px(gf), qy = py(gf), qz = pz(gf);
    AxisList X = axis_list(I, gf.m, qx), Y = axis_list(J, gf.n, qy), Z = axis_list(K, gf.o, qz);
    for (int c = 0; c < Z.n; c++)
        for (int b = 0; b < Y.n; b++)
            for (int a = 0; a < X.n; a++) {
                int ti = 2 * X.C[a] + X.d[a], tj = 2 * Y.C[b] + Y.d[b], tk = 2 * Z.C[c] + Z.d[c];
                const int8_t* fs = Sf + 6 * gf.pi(wrap(ti, gf.m, qx), wrap(tj, gf.n, qy), wrap(tk, gf.o, qz));
                int lo, hi;
                lo = fs[0] + ti; hi = fs[1] + ti; grid_map(lo, hi, gf.m, qx);
                s[0] = min(s[0], lo - I); s[1] = max(s[1], hi - I);
                lo = fs[2] + tj; hi = fs[3] + tj; grid_map(lo, hi, gf.n, qy);
                s[2] = min(s[2], lo - J); s[3] = max(s[3], hi - J);
                lo = fs[4] + tk; hi = fs[5] + tk; grid_map(lo, hi, gf.o, qz);
                s[4] = min(s[4], lo - K); s[5] = max(s[5], hi - K);
            }
    for (int u = 0; u < 6; u++) Sc[6 * q + u] = (int8_t)s[u];
}

// compute_rats (region.cc:629-660) as a gather per coarse point, in the
// reference's accumulation order: fine points in cube scan order (z, y, x
// cubes; x-fastest roles); for each, A_red (:1117-1166) forms
// At(J) = sum_u 0.125*A_f(t,u)*w(u->J) over u in igrid_map's range cropped to
// t's box (kk, jj, ii order), A_mul scales it by 1/2 per non-snapped upper
// axis, and A_add (:1173-1180) adds it to this coarse point's row.  Products
// by powers of two are exact, sums are rounded one by one (no fused
// multiply-add), so the result matches the reference bit for bit.
// One thread per coarse point.  Output: colour-major coarse stencils.
constexpr int kRatBlock = 256;

// The general gather, for any coarse point (boundaries, snapped cubes,
// periodic images, cropped boxes).  Each fine point's 27 coefficients are
// loaded at once into the thread's column `my` of a shared-memory tile (27
// independent loads, one memory latency) and its terms read them there.
static __device__ __noinline__ void rat_general(const LevelGeom& gf, const double* __restrict__ Af,
                                         const int8_t* __restrict__ Sf, int I, int J, int K, double* my,
                                         double* acc) {
    const bool qx = px(gf), qy = py(gf), qz = pz(gf);
    int lx = cube_last(gf.m, qx), ly = cube_last(gf.n, qy), lz = cube_last(gf.o, qz);
    for (int cz = K - 1; cz <= K; cz++) {
        if (cz < cube_first(gf.o, qz) || cz > lz) continue;
        for (int cy = J - 1; cy <= J; cy++) {
            if (cy < cube_first(gf.n, qy) || cy > ly) continue;
            for (int cx = I - 1; cx <= I; cx++) {
                if (cx < cube_first(gf.m, qx) || cx > lx) continue;
                for (int dz = 0; dz < 2; dz++) {
                    if (dz && !has_upper(cz, gf.o, qz)) continue;
                    bool zsn = snapped(cz, gf.o, qz);
                    if (tweight(cz, dz, K, zsn) == 0.0) continue;
                    for (int dy = 0; dy < 2; dy++) {
                        if (dy && !has_upper(cy, gf.n, qy)) continue;
                        bool ysn = snapped(cy, gf.n, qy);
                        if (tweight(cy, dy, J, ysn) == 0.0) continue;
                        for (int dx = 0; dx < 2; dx++) {
                            if (dx && !has_upper(cx, gf.m, qx)) continue;
                            bool xsn = snapped(cx, gf.m, qx);
                            if (tweight(cx, dx, I, xsn) == 0.0) continue;
                            double fac = ((dx && !xsn) ? 0.5 : 1.0) * ((dy && !ysn) ? 0.5 : 1.0) *
                                         ((dz && !zsn) ? 0.5 : 1.0);
                            int ti = 2 * cx + dx, tj = 2 * cy + dy, tk = 2 * cz + dz;
                            int wi = wrap(ti, gf.m, qx), wj = wrap(tj, gf.n, qy), wk = wrap(tk, gf.o, qz);
                            const int8_t* fs = Sf + 6 * gf.pi(wi, wj, wk);
                            int B[6] = {fs[0] + ti, fs[1] + ti, fs[2] + tj, fs[3] + tj, fs[4] + tk, fs[5] + tk};
                            int St[6] = {B[0], B[1], B[2], B[3], B[4], B[5]};
                            grid_map(St[0], St[1], gf.m, qx);
                            grid_map(St[2], St[3], gf.n, qy);
                            grid_map(St[4], St[5], gf.o, qz);
                            int fcol = gf.colour(wi, wj, wk);
                            const double* fa = Af + (long)fcol * 27 * gf.Nc + gf.cidx(wi, wj, wk);
#pragma unroll
                            for (int u = 0; u < 27; u++) my[u * kRatBlock] = __ldg(fa + u * gf.Nc);
                            for (int vk = St[4]; vk < St[5]; vk++) {
                                int lk, uk, ck = igrid_map(lk, uk, B[4], B[5], vk, gf.o, qz);
                                for (int vj = St[2]; vj < St[3]; vj++) {
                                    int lj, uj, cj = igrid_map(lj, uj, B[2], B[3], vj, gf.n, qy);
                                    for (int vi = St[0]; vi < St[1]; vi++) {
                                        int li, ui, ci = igrid_map(li, ui, B[0], B[1], vi, gf.m, qx);
                                        double At = 0.0;
                                        for (int kk = lk; kk < uk; kk++) {
                                            double kfac = kk == ck ? 1.0 : 0.5;
                                            for (int jj = lj; jj < uj; jj++) {
                                                double jkfac = jj == cj ? kfac : 0.5 * kfac;
                                                for (int ii = li; ii < ui; ii++) {
                                                    int slot = (ii - ti + 1) + 3 * (jj - tj + 1) + 9 * (kk - tk + 1);
                                                    double term = __dmul_rn(__dmul_rn(0.125, my[slot * kRatBlock]),
                                                                            ii == ci ? jkfac : 0.5 * jkfac);
                                                    At = __dadd_rn(At, term);
                                                }
                                            }
                                        }
                                        int s = (vi - I + 1) + 3 * (vj - J + 1) + 9 * (vk - K + 1);
                                        acc[s] = __dadd_rn(acc[s], __dmul_rn(At, fac));
                                    }
                                }
                            }
                        }
                    }
                }
            }
        }
    }
}

// The interior gather.  A coarse point of a non-periodic level that is
// interior on every axis (inner_axis: fine points 2I-1, 2I, 2I+1 transfer
// with weights 1/2, 1, 1/2) and whose 27 fine points all have the full box
// [-1,2)^3 takes rat_general's path with every bound, weight and slot known
// at compile time: per axis a fine point at offset o from 2I reaches coarse
// offsets v in [-1,1) (o = -1), [-1,2) (o = 0) or [0,2) (o = 1), gathering
// fine offsets [2v-1, 2v+2) cropped to its box [o-1, o+2); igrid_map's
// coincident point is 2v.  The fine points are visited in the same scan order,
// each At sums its terms in the same (kk, jj, ii) order and each accumulator
// receives the same additions in the same order, so the result is rat_general's
// bit for bit.  With no data-dependent control flow the fine point's 27
// coefficients stay in registers and its At sums are independent chains the
// scheduler can interleave; the 27 accumulators live in the thread's column
// of the shared-memory tile (in registers, beside the coefficients and the
// chains in flight, they spill).
struct RatScan {
    int o[27][3];
};
__host__ __device__ constexpr RatScan rat_scan() {
    RatScan r{};
    int n = 0;
    for (int az = 0; az < 2; az++)
        for (int ay = 0; ay < 2; ay++)
            for (int ax = 0; ax < 2; ax++)
                for (int dz = 0; dz < 2; dz++)
                    for (int dy = 0; dy < 2; dy++)
                        for (int dx = 0; dx < 2; dx++) {
                            const int oz = 2 * az + dz - 2, oy = 2 * ay + dy - 2, ox = 2 * ax + dx - 2;
                            if (ox < -1 || oy < -1 || oz < -1) continue;
                            r.o[n][0] = ox;
                            r.o[n][1] = oy;
                            r.o[n][2] = oz;
                            n++;
                        }
    return r;
}
__host__ __device__ constexpr int rat_imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int rat_imin(int a, int b) { return a < b ? a : b; }

template <int OX, int OY, int OZ>
__device__ __forceinline__ void rat_fast_fine(const double* __restrict__ fa, long nc, double* acc) {
    double h[27];
#pragma unroll
    for (int u = 0; u < 27; u++) h[u] = __dmul_rn(0.125, __ldg(fa + u * nc));
    constexpr double fac = (OX ? 0.5 : 1.0) * (OY ? 0.5 : 1.0) * (OZ ? 0.5 : 1.0);
#pragma unroll
    for (int vz = (OZ == 1 ? 0 : -1); vz < (OZ == -1 ? 1 : 2); vz++)
#pragma unroll
        for (int vy = (OY == 1 ? 0 : -1); vy < (OY == -1 ? 1 : 2); vy++)
#pragma unroll
            for (int vx = (OX == 1 ? 0 : -1); vx < (OX == -1 ? 1 : 2); vx++) {
                double At = 0.0;
#pragma unroll
                for (int kk = rat_imax(2 * vz - 1, OZ - 1); kk < rat_imin(2 * vz + 2, OZ + 2); kk++) {
                    const double kfac = kk == 2 * vz ? 1.0 : 0.5;
#pragma unroll
                    for (int jj = rat_imax(2 * vy - 1, OY - 1); jj < rat_imin(2 * vy + 2, OY + 2); jj++) {
                        const double jkfac = jj == 2 * vy ? kfac : 0.5 * kfac;
#pragma unroll
                        for (int ii = rat_imax(2 * vx - 1, OX - 1); ii < rat_imin(2 * vx + 2, OX + 2); ii++) {
                            const int slot = (ii - OX + 1) + 3 * (jj - OY + 1) + 9 * (kk - OZ + 1);
                            At = __dadd_rn(At, __dmul_rn(h[slot], ii == 2 * vx ? jkfac : 0.5 * jkfac));
                        }
                    }
                }
                const int s = (vx + 1) + 3 * (vy + 1) + 9 * (vz + 1);
                acc[s * kRatBlock] = __dadd_rn(acc[s * kRatBlock], __dmul_rn(At, fac));
            }
}

// Fine point n (0..26, scan order) of the interior gather.  Called from a
// loop that is not unrolled, so the compiler does not hoist the loads of
// later fine points into this one's registers.
template <int N>
__device__ __forceinline__ void rat_fast_step(int n, const LevelGeom& gf, const double* __restrict__ Af, int I,
                                              int J, int K, double* acc) {
    constexpr RatScan R = rat_scan();
    constexpr int OX = R.o[N][0], OY = R.o[N][1], OZ = R.o[N][2];
    if (n == N) {
        const int ti = 2 * I + OX, tj = 2 * J + OY, tk = 2 * K + OZ;
        rat_fast_fine<OX, OY, OZ>(Af + (long)gf.colour(ti, tj, tk) * 27 * gf.Nc + gf.cidx(ti, tj, tk), gf.Nc,
                                  acc);
        return;
    }
    if constexpr (N + 1 < 27) rat_fast_step<N + 1>(n, gf, Af, I, J, K, acc);
}

// Whether an interior coarse point (I,J,K) (CoarseSplit) takes the interior
// gather: all 27 fine boxes [-1,2)^3 (each box is six int8 at an even
// offset, read as three 16-bit words (lo, hi) = (-1, 2)).
__device__ __forceinline__ bool rat_full_boxes(const LevelGeom& gf, const int8_t* __restrict__ Sf, int I, int J,
                                               int K) {
    bool full = true;
#pragma unroll
    for (int oz = -1; oz <= 1; oz++)
#pragma unroll
        for (int oy = -1; oy <= 1; oy++)
#pragma unroll
            for (int ox = -1; ox <= 1; ox++) {
                const uint16_t* b =
                    reinterpret_cast<const uint16_t*>(Sf + 6 * gf.pi(2 * I + ox, 2 * J + oy, 2 * K + oz));
                full = full && __ldg(b) == 0x02FFu && __ldg(b + 1) == 0x02FFu && __ldg(b + 2) == 0x02FFu;
            }
    return full;
}

// Coarse points in CoarseSplit order: the interior box first, whose blocks
// walk the 27 fine points in lock step (a barrier after each), so that the
// warps of an SM run one fine point's code at a time -- unrolled, the 27
// fine points are ~100 KB of instructions, which warps at different fine
// points would keep evicting from the instruction cache -- then the shell,
// whose points take rat_general in warps of their own (mixed into interior
// warps, one boundary point made its whole warp wait for the general path).
// Dynamic shared memory: kRatSmem (the accumulators or the coefficient
// columns, one column of 27 per thread).
constexpr size_t kRatSmem = 27 * kRatBlock * sizeof(double);

static __global__ void __launch_bounds__(kRatBlock, 2) k_rat_fill(LevelGeom gf, LevelGeom gc, CoarseSplit sp,
                                                        const double* __restrict__ Af,
                                                        const int8_t* __restrict__ Sf, double* __restrict__ Ac) {
    extern __shared__ double sa[];
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const bool valid = q < gc.npts;
    int I = 0, J = 0, K = 0;
    const bool inner = valid && split_point(gc, sp, q, I, J, K);
    const bool fast = inner && rat_full_boxes(gf, Sf, I, J, K);
    double* col = sa + threadIdx.x;  // this thread's column: element s at col[s * kRatBlock]
    double* out = nullptr;
    if (valid) out = Ac + (long)gc.colour(I, J, K) * 27 * gc.Nc + gc.cidx(I, J, K);
    if (__syncthreads_or(fast)) {
        if (fast)
            for (int s = 0; s < 27; s++) col[s * kRatBlock] = 0.0;
#pragma unroll 1
        for (int n = 0; n < 27; n++) {
            if (fast) rat_fast_step<0>(n, gf, Af, I, J, K, col);
            __syncthreads();
        }
        if (fast)
            for (int s = 0; s < 27; s++) out[(long)s * gc.Nc] = col[s * kRatBlock];
    }
    if (valid && !fast) {
        double acc[27];
        for (int s = 0; s < 27; s++) acc[s] = 0.0;
        rat_general(gf, Af, Sf, I, J, K, col, acc);
        for (int s = 0; s < 27; s++) out[(long)s * gc.Nc] = acc[s];
    }
}

// k_rat_fill for small coarse levels, where one thread per coarse point
// leaves the GPU nearly empty: one warp per coarse point, lane s < 27 owning
// coarse stencil slot s (neighbour v = (I,J,K) + (s%3-1, s/3%3-1, s/9-1)).
// The warp walks the fine points in scan order together -- their boxes and
// factors are the same for every lane; lanes 0..26 first load the fine
// point's 27 coefficients into the warp's shared row -- and each lane adds
// the term for its own v, so every accumulator receives its terms in the
// same order as in k_rat_fill: the results are identical.
constexpr int kRatSmallBlock = 128;
constexpr long kRatSmallMax = 20000;  // coarse levels up to this size use the warp form

static __global__ void __launch_bounds__(kRatSmallBlock, 4) k_rat_fill_small(LevelGeom gf, LevelGeom gc,
                                                                   const double* __restrict__ Af,
                                                                   const int8_t* __restrict__ Sf,
                                                                   double* __restrict__ Ac) {
    __shared__ double srow[kRatSmallBlock / 32][32];
    long q = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    double* row = srow[threadIdx.x >> 5];
    if (q >= gc.npts) return;
    int I, J, K;
    decode_nat(gc, q, I, J, K);
    const bool mine = lane < 27;
    const int vi = I + lane % 3 - 1, vj = J + (lane / 3) % 3 - 1, vk = K + lane / 9 - 1;
    double acc = 0.0;
    const bool qx = px(gf), qy = py(gf), qz = pz(gf);
    int lx = cube_last(gf.m, qx), ly = cube_last(gf.n, qy), lz = cube_last(gf.o, qz);
    for (int cz = K - 1; cz <= K; cz++) {
        if (cz < cube_first(gf.o, qz) || cz > lz) continue;
        for (int cy = J - 1; cy <= J; cy++) {
            if (cy < cube_first(gf.n, qy) || cy > ly) continue;
            for (int cx = I - 1; cx <= I; cx++) {
                if (cx < cube_first(gf.m, qx) || cx > lx) continue;
                for (int dz = 0; dz < 2; dz++) {
                    if (dz && !has_upper(cz, gf.o, qz)) continue;
                    bool zsn = snapped(cz, gf.o, qz);
                    if (tweight(cz, dz, K, zsn) == 0.0) continue;
                    for (int dy = 0; dy < 2; dy++) {
                        if (dy && !has_upper(cy, gf.n, qy)) continue;
                        bool ysn = snapped(cy, gf.n, qy);
                        if (tweight(cy, dy, J, ysn) == 0.0) continue;
                        for (int dx = 0; dx < 2; dx++) {
                            if (dx && !has_upper(cx, gf.m, qx)) continue;
                            bool xsn = snapped(cx, gf.m, qx);
                            if (tweight(cx, dx, I, xsn) == 0.0) continue;
                            double fac = ((dx && !xsn) ? 0.5 : 1.0) * ((dy && !ysn) ? 0.5 : 1.0) *
                                         ((dz && !zsn) ? 0.5 : 1.0);
                            int ti = 2 * cx + dx, tj = 2 * cy + dy, tk = 2 * cz + dz;
                            int wi = wrap(ti, gf.m, qx), wj = wrap(tj, gf.n, qy), wk = wrap(tk, gf.o, qz);
                            const double* fa = Af + (long)gf.colour(wi, wj, wk) * 27 * gf.Nc + gf.cidx(wi, wj, wk);
                            __syncwarp();
                            if (mine) row[lane] = __ldg(fa + lane * gf.Nc);
                            __syncwarp();
                            const int8_t* fs = Sf + 6 * gf.pi(wi, wj, wk);
                            int B[6] = {fs[0] + ti, fs[1] + ti, fs[2] + tj, fs[3] + tj, fs[4] + tk, fs[5] + tk};
                            int St[6] = {B[0], B[1], B[2], B[3], B[4], B[5]};
                            grid_map(St[0], St[1], gf.m, qx);
                            grid_map(St[2], St[3], gf.n, qy);
                            grid_map(St[4], St[5], gf.o, qz);
                            if (!mine || vi < St[0] || vi >= St[1] || vj < St[2] || vj >= St[3] || vk < St[4] ||
                                vk >= St[5])
                                continue;
                            int lk, uk, ck = igrid_map(lk, uk, B[4], B[5], vk, gf.o, qz);
                            int lj, uj, cj = igrid_map(lj, uj, B[2], B[3], vj, gf.n, qy);
                            int li, ui, ci = igrid_map(li, ui, B[0], B[1], vi, gf.m, qx);
                            double At = 0.0;
                            for (int kk = lk; kk < uk; kk++) {
                                double kfac = kk == ck ? 1.0 : 0.5;
                                for (int jj = lj; jj < uj; jj++) {
                                    double jkfac = jj == cj ? kfac : 0.5 * kfac;
                                    for (int ii = li; ii < ui; ii++) {
                                        int slot = (ii - ti + 1) + 3 * (jj - tj + 1) + 9 * (kk - tk + 1);
                                        double term = __dmul_rn(__dmul_rn(0.125, row[slot]),
                                                                ii == ci ? jkfac : 0.5 * jkfac);
                                        At = __dadd_rn(At, term);
                                    }
                                }
                            }
                            acc = __dadd_rn(acc, __dmul_rn(At, fac));
                        }
                    }
                }
            }
        }
    }
    if (mine) Ac[((long)gc.colour(I, J, K) * 27 + lane) * gc.Nc + gc.cidx(I, J, K)] = acc;
}

// k_rat_fill restructured for throughput on non-periodic levels: one thread
// per (coarse point, coarse stencil slot) -- the accumulator of that slot in
// a register -- and the fine stencils and boxes the coarse points read staged
// in shared memory once per CTA instead of per thread.  A CTA covers kRtX
// coarse points of one coarse row (threads: slot-major, so a warp is 32
// consecutive coarse points with the same slot and the same control flow in
// the interior) and walks up kRtKC coarse planes; the fine points that
// transfer to them lie in fine rows 2J-1..2J+1 and fine x 2*I0-1..2*I0+63,
// held as a ring of three fine planes.  Each accumulator receives k_rat_fill's
// terms in k_rat_fill's order (fine points in cube scan order, each fine
// point's terms in A_red's order), so the coarse stencils are the same bit
// for bit.
constexpr int kRtX = 32;
constexpr int kRtThreads = kRtX * 27;
constexpr int kRtKC = 16;
constexpr int kRtFX = 2 * kRtX + 2;  // 65 fine x values, padded
constexpr int kRtPA = 27 * 3 * kRtFX;  // doubles per staged fine plane
constexpr int kRtPS = 3 * kRtFX * 8;   // box bytes per staged fine plane
constexpr size_t kRtSmem = 3 * (kRtPA * sizeof(double) + kRtPS);

static __global__ void __launch_bounds__(kRtThreads, 1) k_rat_tile(LevelGeom gf, LevelGeom gc,
                                                                   const double* __restrict__ Af,
                                                                   const int8_t* __restrict__ Sf,
                                                                   double* __restrict__ Ac) {
    extern __shared__ double rsm[];
    double* As = rsm;
    int8_t* Ss = reinterpret_cast<int8_t*>(rsm + 3 * kRtPA);
    const int I0 = blockIdx.x * kRtX, J = blockIdx.y, K0 = blockIdx.z * kRtKC;
    const int K1 = K0 + kRtKC < gc.o ? K0 + kRtKC : gc.o;
    const int fi0 = 2 * I0 - 1, fj0 = 2 * J - 1;
    const int tid = threadIdx.x;
    const int slot = tid / kRtX;
    const int I = I0 + tid % kRtX;
    auto stage = [&](int fk) {
        if (fk < 0 || fk >= gf.o) return;
        double* A = As + (fk % 3) * kRtPA;
        int8_t* S = Ss + (fk % 3) * kRtPS;
        for (int e = tid; e < 27 * 3 * 65; e += kRtThreads) {
            int fx = e % 65, t2 = e / 65, fy = t2 % 3, q = t2 / 3;
            int fi = fi0 + fx, fj = fj0 + fy;
            if (fi < 0 || fi >= gf.m || fj < 0 || fj >= gf.n) continue;
            A[(q * 3 + fy) * kRtFX + fx] = __ldg(Af + gf.ai(fi, fj, fk, q));
        }
        for (int e = tid; e < 3 * 65 * 6; e += kRtThreads) {
            int u = e % 6, t2 = e / 6, fx = t2 % 65, fy = t2 / 65;
            int fi = fi0 + fx, fj = fj0 + fy;
            if (fi < 0 || fi >= gf.m || fj < 0 || fj >= gf.n) continue;
            S[(fy * kRtFX + fx) * 8 + u] = Sf[6 * gf.pi(fi, fj, fk) + u];
        }
    };
    const int vi = I + slot % 3 - 1, vj = J + (slot / 3) % 3 - 1;
    const int lx = cube_last(gf.m), ly = cube_last(gf.n), lz = cube_last(gf.o);
    stage(2 * K0 - 1);
    for (int K = K0; K < K1; K++) {
        stage(2 * K);
        stage(2 * K + 1);
        __syncthreads();
        const int vk = K + slot / 9 - 1;
        if (I < gc.m) {
            double acc = 0.0;
            for (int cz = K - 1; cz <= K; cz++) {
                if (cz < 0 || cz > lz) continue;
                for (int cy = J - 1; cy <= J; cy++) {
                    if (cy < 0 || cy > ly) continue;
                    for (int cx = I - 1; cx <= I; cx++) {
                        if (cx < 0 || cx > lx) continue;
                        for (int dz = 0; dz < 2; dz++) {
                            if (dz && !has_upper(cz, gf.o)) continue;
                            bool zsn = snapped(cz, gf.o);
                            if (tweight(cz, dz, K, zsn) == 0.0) continue;
                            for (int dy = 0; dy < 2; dy++) {
                                if (dy && !has_upper(cy, gf.n)) continue;
                                bool ysn = snapped(cy, gf.n);
                                if (tweight(cy, dy, J, ysn) == 0.0) continue;
                                for (int dx = 0; dx < 2; dx++) {
                                    if (dx && !has_upper(cx, gf.m)) continue;
                                    bool xsn = snapped(cx, gf.m);
                                    if (tweight(cx, dx, I, xsn) == 0.0) continue;
                                    double fac = ((dx && !xsn) ? 0.5 : 1.0) * ((dy && !ysn) ? 0.5 : 1.0) *
                                                 ((dz && !zsn) ? 0.5 : 1.0);
                                    int ti = 2 * cx + dx, tj = 2 * cy + dy, tk = 2 * cz + dz;
                                    const int fx = ti - fi0, fy = tj - fj0;
                                    const int8_t* fs = Ss + (tk % 3) * kRtPS + (fy * kRtFX + fx) * 8;
                                    int B[6] = {fs[0] + ti, fs[1] + ti, fs[2] + tj, fs[3] + tj, fs[4] + tk, fs[5] + tk};
                                    int St[6] = {B[0], B[1], B[2], B[3], B[4], B[5]};
                                    grid_map(St[0], St[1], gf.m);
                                    grid_map(St[2], St[3], gf.n);
                                    grid_map(St[4], St[5], gf.o);
                                    if (vi < St[0] || vi >= St[1] || vj < St[2] || vj >= St[3] || vk < St[4] ||
                                        vk >= St[5])
                                        continue;
                                    const double* row = As + (tk % 3) * kRtPA + fy * kRtFX + fx;
                                    int lk, uk, ck = igrid_map(lk, uk, B[4], B[5], vk, gf.o);
                                    int lj, uj, cj = igrid_map(lj, uj, B[2], B[3], vj, gf.n);
                                    int li, ui, ci = igrid_map(li, ui, B[0], B[1], vi, gf.m);
                                    double At = 0.0;
                                    for (int kk = lk; kk < uk; kk++) {
                                        double kfac = kk == ck ? 1.0 : 0.5;
                                        for (int jj = lj; jj < uj; jj++) {
                                            double jkfac = jj == cj ? kfac : 0.5 * kfac;
                                            for (int ii = li; ii < ui; ii++) {
                                                int q = (ii - ti + 1) + 3 * (jj - tj + 1) + 9 * (kk - tk + 1);
                                                double term = __dmul_rn(__dmul_rn(0.125, row[q * 3 * kRtFX]),
                                                                        ii == ci ? jkfac : 0.5 * jkfac);
                                                At = __dadd_rn(At, term);
                                            }
                                        }
                                    }
                                    acc = __dadd_rn(acc, __dmul_rn(At, fac));
                                }
                            }
                        }
                    }
                }
            }
            Ac[((long)gc.colour(I, J, K) * 27 + slot) * gc.Nc + gc.cidx(I, J, K)] = acc;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Coarsest level: dense column-major matrix Aexact[row + col*n] from the
// level's stencils (region_tr.cc:489-508, non-periodic: no wrap needed).
static __global__ void k_lu_build(LevelGeom g, const double* __restrict__ A, const int8_t* __restrict__ S,
                                  double* __restrict__ M) {
    // One thread per row, the box's entries in box order (dk, dj, di
    // ascending), column indices wrapped on periodic axes (step_mod,
    // region.hh:466); an entry is assigned, so when two entries of a row wrap
    // onto one column (a periodic axis of size 1 or 2) the later one stays,
    // as in the reference.
    long row = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long n = g.npts;
    if (row >= n) return;
    int i = (int)(row % g.m); long t = row / g.m; int j = (int)(t % g.n); int k = (int)(t / g.n);
    const int8_t* b = S + 6 * row;
    for (int dk = b[4]; dk < b[5]; dk++)
        for (int dj = b[2]; dj < b[3]; dj++)
            for (int di = b[0]; di < b[1]; di++) {
                int ii = i + di, jj = j + dj, kk = k + dk;
                ii = ii < 0 ? ii + g.m : (ii >= g.m ? ii - g.m : ii);
                jj = jj < 0 ? jj + g.n : (jj >= g.n ? jj - g.n : jj);
                kk = kk < 0 ? kk + g.o : (kk >= g.o ? kk - g.o : kk);
                int s = (di + 1) + 3 * (dj + 1) + 9 * (dk + 1);
                M[row + g.pi(ii, jj, kk) * n] = A[g.ai(i, j, k, s)];
            }
}

// Explicit inverse from the factors: column c of Minv (row-major) solves
// A x = e_c as P e_c, then L y = b and U x = y, column-oriented.  One thread
// block per column, the vector in shared memory; at step j every entry below
// (forward) or above (backward) j is updated in parallel, each entry
// receiving the same sequence of operations, in the same order, as a
// sequential column solve would apply -- so the result does not depend on
// the block size.
static __global__ void __launch_bounds__(256) k_lu_inverse(const double* __restrict__ M, const int* __restrict__ piv,
                                                    int n, double* __restrict__ Minv) {
    extern __shared__ double X[];
    int c = blockIdx.x;
    for (int i = threadIdx.x; i < n; i += blockDim.x) X[i] = (i == c) ? 1.0 : 0.0;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = 0; i < n; i++) {
            int p = piv[i] - 1;
            if (p != i) {
                double t = X[i];
                X[i] = X[p];
                X[p] = t;
            }
        }
    __syncthreads();
    for (int j = 0; j < n; j++) {
        double xj = X[j];
        if (xj != 0.0)
            for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x)
                X[i] = __dsub_rn(X[i], __dmul_rn(xj, M[i + (long)j * n]));
        __syncthreads();
    }
    for (int j = n - 1; j >= 0; j--) {
        double xj = X[j];
        if (xj != 0.0) {
            xj = xj / M[j + (long)j * n];
            for (int i = threadIdx.x; i < j; i += blockDim.x)
                X[i] = __dsub_rn(X[i], __dmul_rn(xj, M[i + (long)j * n]));
        }
        if (threadIdx.x == 0) Minv[(long)j * n + c] = xj;
        __syncthreads();
    }
}

// Widest extent of the factors' non-zeros off the diagonal, for
// k_lu_inverse_band: ext[0] = max over columns j of (last row i > j with
// M(i,j) != 0) - j, ext[1] = max of j - (first row i < j with M(i,j) != 0);
// ext zeroed by the caller.  One warp per column.
static __global__ void __launch_bounds__(256) k_lu_extent(const double* __restrict__ M, int n, int* __restrict__ ext) {
    const int j = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (j >= n) return;
    int lo = 0, up = 0;
    const double* col = M + (long)j * n;
    for (int i = lane; i < n; i += 32)
        if (col[i] != 0.0) {
            if (i > j) lo = max(lo, i - j);
            else if (i < j) up = max(up, j - i);
        }
    for (int o = 16; o > 0; o >>= 1) {
        lo = max(lo, __shfl_down_sync(0xffffffffu, lo, o));
        up = max(up, __shfl_down_sync(0xffffffffu, up, o));
    }
    if (lane == 0) {
        atomicMax(ext, lo);
        atomicMax(ext + 1, up);
    }
}

// k_lu_inverse with one warp per column and the factors' band: at forward
// step j the entries below j within bl rows, at backward step j those above
// within bu rows (k_lu_extent; everything beyond is zero, and an update by a
// zero factor entry changes no bit of a solution entry, which can never be
// -0 here), each entry receiving the same operations in the same order as in
// k_lu_inverse -- the same inverse bit for bit.  A warp works through its
// column without block barriers, loading the factor entries of several steps
// at once so that their L2 latency is paid once per group of steps; the
// 729 columns of a 9^3 level run as 729 concurrent warps.  A lane holds RL
// rows of the forward band (bl <= 32 RL) for GF steps at a time and 8 rows
// of the backward band (bu <= 256) for 4 steps.  Dynamic shared memory:
// kInvWarps columns of n doubles.
constexpr int kInvWarps = 4;
constexpr int kInvGroupB = 4;

template <int RL, int GF>
__global__ void __launch_bounds__(32 * kInvWarps) k_lu_inverse_band(const double* __restrict__ M,
                                                                      const int* __restrict__ piv, int n, int bl,
                                                                      int bu, double* __restrict__ Minv) {
    extern __shared__ double Xs[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * kInvWarps + w;
    if (c >= n) return;  // a whole warp; no block barrier follows
    double* X = Xs + (size_t)w * n;
    for (int i = lane; i < n; i += 32) X[i] = i == c ? 1.0 : 0.0;
    __syncwarp();
    if (lane == 0)
        for (int i = 0; i < n; i++) {
            const int p = piv[i] - 1;
            if (p != i) {
                const double t = X[i];
                X[i] = X[p];
                X[p] = t;
            }
        }
    __syncwarp();
    for (int j0 = 0; j0 < n; j0 += GF) {
        double Lb[GF][RL];
#pragma unroll
        for (int s = 0; s < GF; s++)
#pragma unroll
            for (int k = 0; k < RL; k++) {
                const int j = j0 + s, a = lane + 32 * k, i = j + 1 + a;
                Lb[s][k] = (j < n && a < bl && i < n) ? M[i + (long)j * n] : 0.0;
            }
#pragma unroll
        for (int s = 0; s < GF; s++) {
            const int j = j0 + s;
            if (j < n) {
                const double xj = X[j];
                if (xj != 0.0)
#pragma unroll
                    for (int k = 0; k < RL; k++) {
                        const int a = lane + 32 * k, i = j + 1 + a;
                        if (a < bl && i < n) X[i] = __dsub_rn(X[i], __dmul_rn(xj, Lb[s][k]));
                    }
            }
            __syncwarp();
        }
    }
    for (int j0 = n - 1; j0 >= 0; j0 -= kInvGroupB) {
        double Ub[kInvGroupB][8], dg[kInvGroupB];
#pragma unroll
        for (int s = 0; s < kInvGroupB; s++) {
            const int j = j0 - s;
            dg[s] = j >= 0 ? M[j + (long)j * n] : 1.0;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int a = lane + 32 * k, i = j - 1 - a;
                Ub[s][k] = (j >= 0 && a < bu && i >= 0) ? M[i + (long)j * n] : 0.0;
            }
        }
#pragma unroll
        for (int s = 0; s < kInvGroupB; s++) {
            const int j = j0 - s;
            if (j >= 0) {
                double xj = X[j];
                if (xj != 0.0) {
                    xj = xj / dg[s];
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        const int a = lane + 32 * k, i = j - 1 - a;
                        if (a < bu && i >= 0) X[i] = __dsub_rn(X[i], __dmul_rn(xj, Ub[s][k]));
                    }
                }
                if (lane == 0) Minv[(long)j * n + c] = xj;
            }
            __syncwarp();
        }
    }
}

// Coarse solve by the explicit inverse: x(i) = sum_c Minv[i][c] * r(c), one
// warp per row, FP64 accumulation, fixed reduction tree.  r is the level's
// colour-major source (type T), x its halo'd solution.
template <class T>
static __global__ void __launch_bounds__(256) k_lu_apply(LevelGeom g, const double* __restrict__ Minv,
                                                  const T* __restrict__ r, T* __restrict__ x) {
    pdl_enter();
    int n = (int)g.npts;
    int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int l = threadIdx.x & 31;
    if (row >= n) return;
    double s = 0.0;
    for (int c = l; c < n; c += 32) {
        int i = c % g.m, t = c / g.m, j = t % g.n, k = t / g.n;
        s = fma(Minv[(long)row * n + c], (double)r[g.ri(i, j, k)], s);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (l == 0) {
        int i = row % g.m, t = row / g.m, j = t % g.n, k = t / g.n;
        x[g.xi(i, j, k)] = (T)s;
    }
}

// Coarse solve in DGETRS order (one block): the interchanges, then
// column-oriented forward and backward substitution, each column's updates
// in parallel -- the same operations as the oracle's restatement, so the
// result matches it bit for bit.  buf: n doubles of scratch.
template <class T>
static __global__ void __launch_bounds__(1024) k_lu_solve_exact(LevelGeom g, const double* __restrict__ M,
                                                         const int* __restrict__ piv, const T* __restrict__ r,
                                                         T* __restrict__ x, double* __restrict__ b) {
    pdl_enter();
    int n = (int)g.npts;
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
        int i = c % g.m, t = c / g.m, j = t % g.n, k = t / g.n;
        b[c] = (double)r[g.ri(i, j, k)];
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = 0; i < n; i++) {
            int p = piv[i] - 1;
            if (p != i) { double t = b[i]; b[i] = b[p]; b[p] = t; }
        }
    __syncthreads();
    for (int j = 0; j < n; j++) {
        double xj = b[j];
        if (xj != 0.0)
            for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) b[i] = __dsub_rn(b[i], __dmul_rn(xj, M[i + (long)j * n]));
        __syncthreads();
    }
    for (int j = n - 1; j >= 0; j--) {
        double xj = b[j];
        if (xj != 0.0) {
            xj = xj / M[j + (long)j * n];
            for (int i = threadIdx.x; i < j; i += blockDim.x) b[i] = __dsub_rn(b[i], __dmul_rn(xj, M[i + (long)j * n]));
        }
        __syncthreads();
        if (threadIdx.x == 0 && xj != 0.0) b[j] = xj;
        __syncthreads();
    }
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
        int i = c % g.m, t = c / g.m, j = t % g.n, k = t / g.n;
        x[g.xi(i, j, k)] = (T)b[c];
    }
}

// ---------------------------------------------------------------------------
// Input synthesis on the device (the host generators of problems.cpp, same
// operation order, no fused multiply-add, so the results are bit for bit the
// host arrays):
//   k_assemble_q1: Q1 FEM stencils of -div(kappa grad u) from a cell field
//   (kappa itself, or g with kappa = exp(sigma*g) when from_log), Dirichlet
//   fix rows on the boundary, boxes; written straight into the level-0
//   colour-major stencils.
__device__ __forceinline__ double cell_kappa(const double* c, long idx, int from_log, double sigma) {
    if (!c) return 1.0;
    return from_log ? exp(sigma * c[idx]) : c[idx];
}

// kappa = exp(sigma * g) of every cell, once: k_assemble_q1 reads each
// cell's kappa from its 8 corner points, and evaluating the exponential
// there 8 times over bounded that kernel.  The same expression, so the
// same values as cell_kappa's.
static __global__ void __launch_bounds__(256) k_cell_exp(const double* __restrict__ g, long n, double sigma,
                                                         double* __restrict__ kap) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) kap[i] = exp(sigma * g[i]);
}

static __global__ void __launch_bounds__(128) k_assemble_q1(LevelGeom g, const double* __restrict__ cells, int from_log,
                                                     double sigma, double h, double* __restrict__ A,
                                                     int8_t* __restrict__ S) {
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= g.npts) return;
    int i, j, k;
    decode_nat(g, q, i, j, k);
    long nx = g.m - 1, ny = g.n - 1;
    const double khat[4] = {1.0 / 3.0, 0.0, -1.0 / 12.0, -1.0 / 12.0};
    double c[27];
#pragma unroll
    for (int s = 0; s < 27; s++) c[s] = 0.0;
    bool interior = i > 0 && i < g.m - 1 && j > 0 && j < g.n - 1 && k > 0 && k < g.o - 1;
    if (interior) {
        for (int ce = -1; ce <= 0; ce++)
            for (int cb = -1; cb <= 0; cb++)
                for (int ca = -1; ca <= 0; ca++) {
                    double ke = __dmul_rn(h, cell_kappa(cells, (i + ca) + nx * ((j + cb) + ny * (long)(k + ce)), from_log, sigma));
                    for (int ee = 0; ee < 2; ee++)
                        for (int bb = 0; bb < 2; bb++)
                            for (int aa = 0; aa < 2; aa++) {
                                int diff = (aa != -ca) + (bb != -cb) + (ee != -ce);
                                int s = (aa + ca + 1) + 3 * (bb + cb + 1) + 9 * (ee + ce + 1);
                                c[s] = __dadd_rn(c[s], __dmul_rn(ke, khat[diff]));
                            }
                }
    } else {
        double sum = 0;
        int cnt = 0;
        for (int e = -1; e <= 0; e++)
            for (int b = -1; b <= 0; b++)
                for (int a = -1; a <= 0; a++) {
                    long ci = i + a, cj = j + b, ck = k + e;
                    if (ci < 0 || cj < 0 || ck < 0 || ci >= nx || cj >= ny || ck >= g.o - 1) continue;
                    sum = __dadd_rn(sum, cell_kappa(cells, ci + nx * (cj + ny * ck), from_log, sigma));
                    cnt++;
                }
        c[13] = __dmul_rn(__dmul_rn(8.0 / 3.0, h), __ddiv_rn(sum, (double)cnt));
    }
#pragma unroll
    for (int s = 0; s < 27; s++) A[g.ai(i, j, k, s)] = c[s];
    int8_t* b = S + 6 * q;
    b[0] = b[2] = b[4] = interior ? -1 : 0;
    b[1] = b[3] = b[5] = interior ? 2 : 1;
}

// Right-hand side: interior uniform[-1,1] from SplitMix64(key ^ index), the
// integer recipe of pgmg_problem_rhs, boundary 0; into the colour-major source.
__device__ __forceinline__ uint64_t d_splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static __global__ void __launch_bounds__(256) k_rhs_uniform(LevelGeom g, uint64_t seed, double* __restrict__ r) {
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= g.npts) return;
    int i, j, k;
    decode_nat(g, q, i, j, k);
    uint64_t key = (seed + 0x5851F42D4C957F2Dull) * 0x2545F4914F6CDD1Dull;
    bool interior = i > 0 && i < g.m - 1 && j > 0 && j < g.n - 1 && k > 0 && k < g.o - 1;
    double v = 0.0;
    if (interior) {
        double u = (double)((d_splitmix64(key ^ (uint64_t)q) >> 11) + 1) * (1.0 / 9007199254740992.0);
        v = 2.0 * (u - 0.5);
    }
    r[g.ri(i, j, k)] = v;
}

// ---------------------------------------------------------------------------
// Pivot candidate order of the LU kernels: larger |value|, then the first row.
__device__ __forceinline__ void lu_better(double v, int i, double& bv, int& bi) {
    if (v > bv || (v == bv && i < bi)) { bv = v; bi = i; }
}

// Partial-pivoting LU (DGETF2 order: idamax pivot, row interchange over all
// columns, scaling by the reciprocal pivot, rank-1 update skipping zero
// pivot-row entries) of the coarsest level's dense column-major matrix, in
// one thread block.  The 27-point stencil in natural order gives the matrix
// lower and upper bandwidth kl = ku = 1 + m + m*n; with row interchanges the
// multipliers of column j stay in rows j+1..j+kl and the pivot row in
// columns up to j+kl+ku, so the pivot search, scaling and update run over
// that window only.  Entries outside it are zero and a dense factorisation
// would leave them zero, so the factors are the dense ones bit for bit.
constexpr int kLuBandMax = 2048;

static __global__ void __launch_bounds__(1024) k_lu_band(double* __restrict__ M, int n, int kl, int ku,
                                                  int* __restrict__ piv, int* __restrict__ info) {
    __shared__ double sL[kLuBandMax];
    __shared__ double sU[kLuBandMax];
    __shared__ double wv[32];
    __shared__ int wi[32];
    __shared__ int s_p;
    int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
    if (tid == 0) info[0] = 0;
    for (int j = 0; j < n; j++) {
        int R = min(n - 1, j + kl) - j;       // rows below the diagonal that can be non-zero
        int C = min(n - 1, j + kl + ku) - j;  // columns right of it in the pivot row
        // Pivot: first row of largest |M(i,j)|, i = j..j+R.
        double bv = -1.0;
        int bi = n;
        for (int i = j + tid; i <= j + R; i += blockDim.x) lu_better(fabs(M[i + (long)j * n]), i, bv, bi);
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_down_sync(0xffffffffu, bv, o);
            int oi = __shfl_down_sync(0xffffffffu, bi, o);
            lu_better(ov, oi, bv, bi);
        }
        if (lane == 0) { wv[w] = bv; wi[w] = bi; }
        __syncthreads();
        if (tid == 0) {
            for (int q = 1; q < nw; q++) lu_better(wv[q], wi[q], wv[0], wi[0]);
            int p = wi[0] < n ? wi[0] : j;
            s_p = p;
            piv[j] = p + 1;
        }
        __syncthreads();
        int p = s_p;
        double apj = M[p + (long)j * n];
        if (apj != 0.0) {
            if (p != j)
                for (int c = tid; c < n; c += blockDim.x) {
                    double a = M[j + (long)c * n], b2 = M[p + (long)c * n];
                    M[j + (long)c * n] = b2;
                    M[p + (long)c * n] = a;
                }
            __syncthreads();
            double r = 1.0 / M[j + (long)j * n];
            for (int i = tid; i < R; i += blockDim.x) {
                long a = j + 1 + i + (long)j * n;
                double v = __dmul_rn(M[a], r);
                M[a] = v;
                sL[i] = v;
            }
        } else {
            if (tid == 0 && info[0] == 0) info[0] = j + 1;
            for (int i = tid; i < R; i += blockDim.x) sL[i] = M[j + 1 + i + (long)j * n];
        }
        for (int k = tid; k < C; k += blockDim.x) sU[k] = M[j + (long)(j + 1 + k) * n];
        __syncthreads();
        for (int q = tid; q < R * C; q += blockDim.x) {
            int ii = q % R, kk = q / R;
            double u = sU[kk];
            if (u != 0.0) {
                long a = (j + 1 + ii) + (long)(j + 1 + kk) * n;
                M[a] = __dsub_rn(M[a], __dmul_rn(sL[ii], u));
            }
        }
        __syncthreads();
    }
}

// The same factorisation with the active window in shared memory.  At step
// j only rows j..j+kl and columns j..j+kl+ku can change (above), so the
// kernel keeps that window -- (kl+1) x (kl+ku+1) doubles, rows and columns
// stored circularly (row i in slot i mod (kl+1), column c in slot
// c mod (kl+ku+1), the slots of a step's rows and columns found by counting
// from the step's first slot, never by a division) -- and streams the matrix
// through it: a row or column enters from the dense matrix in the step before
// it is first needed (no earlier step has touched it; its loads are issued at
// the start of that step) and leaves when its entries are final (column j and
// row j, written to the dense matrix in step j).  Per step: the swap, scaling
// and leaving writes; a barrier; the rank-1 update (warp w: columns 1+w,
// 33+w, ...; lanes: rows), the entering row and column, and warp 0's pivot
// search of the next column, which warp 0 has just updated itself; a
// barrier.  The row interchanges' effect on the multipliers already written
// (left of the step's column) is applied at the end, column by column in
// step order, which leaves the same dense factors as interchanging whole
// rows at every step.  Every entry receives k_lu_band's operations in the
// same order, so the factors and pivots are identical.  Needs
// (kl+1) + (kl+ku+1) <= 1024 (one thread per entering entry).
constexpr size_t kLuWindowSmemMax = 220 * 1024;
__host__ __device__ inline size_t lu_window_smem(int n, int kl, int ku) {
    return sizeof(double) * ((size_t)(kl + 1) * (kl + ku + 1) + kl + (kl + ku) + 2) + sizeof(int) * ((size_t)n + 8);
}

static __global__ void __launch_bounds__(1024) k_lu_window(double* __restrict__ M, int n, int kl, int ku,
                                                           int* __restrict__ piv, int* __restrict__ info) {
    extern __shared__ double smem[];
    const int RW = kl + 1, CW = kl + ku + 1;
    double* W = smem;                                    // (i, c) at W[slot(c) * RW + slot(i)]
    double* sL = W + (size_t)RW * CW;                    // the step's multipliers, rows j+1..j+kl
    double* sU = sL + kl;                                // the step's pivot row, columns j+1..j+kl+ku
    double* sv = sU + (kl + ku);                         // [0] the pivot, [1] the diagonal entry before the interchange
    int* pv = reinterpret_cast<int*>(sv + 2);            // pivot row of every step
    int* sp = pv + n;                                    // [0] the step's pivot row
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    if (tid == 0) info[0] = 0;
    for (int e = tid; e < RW * CW; e += blockDim.x) {
        const int c = e / RW, r = e - c * RW;  // at j = 0 slot = index
        W[e] = (r < n && c < n) ? M[r + (long)c * n] : 0.0;
    }
    __syncthreads();
    // Pivot search of column j by warp 0 (rows j..j+R, slots from rs).
    auto pivot = [&](int j, int rs, int cs) {
        const int R = min(n - 1, j + kl) - j;
        double bv = -1.0;
        int bi = n;
        for (int a = lane; a <= R; a += 32) {
            int s = rs + a;
            if (s >= RW) s -= RW;
            lu_better(fabs(W[(size_t)cs * RW + s]), j + a, bv, bi);
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, bv, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            lu_better(ov, oi, bv, bi);
        }
        if (lane == 0) {
            const int p = bi < n ? bi : j;
            int ps = rs + (p - j);
            if (ps >= RW) ps -= RW;
            sp[0] = p;
            sv[0] = W[(size_t)cs * RW + ps];
            sv[1] = W[(size_t)cs * RW + rs];
            pv[j] = p;
            piv[j] = p + 1;
        }
    };
    if (warp == 0) pivot(0, 0, 0);
    __syncthreads();
    int rs0 = 0, cs0 = 0;  // slots of row j and column j
    for (int j = 0; j < n; j++) {
        const int R = min(n - 1, j + kl) - j, C = min(n - 1, j + kl + ku) - j;
        // The row and column entering after this step hold original values:
        // load them now (thread t < CW: entering row, column j+1+t; thread
        // CW + t, t < RW: entering column, row j+1+t).
        const int nr = j + kl + 1, ncl = j + kl + ku + 1;
        double ent = 0.0;
        bool has_ent = false;
        if (tid < CW) {
            const int c = j + 1 + tid;
            has_ent = nr < n && c < n;
            if (has_ent) ent = M[nr + (long)c * n];
        } else if (tid < CW + RW) {
            const int r = j + 1 + (tid - CW);
            has_ent = ncl < n && r < n;
            if (has_ent) ent = M[r + (long)ncl * n];
        }
        // (Read from the pivot search's copies: this phase rewrites both
        // entries of the matrix window.)
        const int p = sp[0];
        int ps = rs0 + (p - j);
        if (ps >= RW) ps -= RW;
        const double apj = sv[0], ajj = sv[1];
        if (apj != 0.0) {
            const double rinv = 1.0 / apj;
            if (tid < C) {
                // column j+1+tid: interchange rows j and p; the pivot row
                // (now row j) is final.
                int cs = cs0 + 1 + tid;
                if (cs >= CW) cs -= CW;
                double* col = W + (size_t)cs * RW;
                const double a = col[rs0], b = col[ps];
                if (p != j) {
                    col[rs0] = b;
                    col[ps] = a;
                }
                sU[tid] = b;
                M[j + (long)(j + 1 + tid) * n] = b;
            } else if (tid < C + R) {
                // row j+1+a of column j: the multiplier (row p holds the old
                // row j's entry after the interchange).
                const int a = tid - C;
                int s = rs0 + 1 + a;
                if (s >= RW) s -= RW;
                const double v = __dmul_rn(j + 1 + a == p ? ajj : W[(size_t)cs0 * RW + s], rinv);
                W[(size_t)cs0 * RW + s] = v;
                sL[a] = v;
                M[(j + 1 + a) + (long)j * n] = v;
            } else if (tid == C + R) {
                W[(size_t)cs0 * RW + rs0] = apj;
                M[j + (long)j * n] = apj;
            }
        } else {
            // Zero pivot (the whole column is zero): no interchange, no
            // scaling, info records the first one.
            if (tid == 0 && info[0] == 0) info[0] = j + 1;
            if (tid < C) {
                int cs = cs0 + 1 + tid;
                if (cs >= CW) cs -= CW;
                const double b = W[(size_t)cs * RW + rs0];
                sU[tid] = b;
                M[j + (long)(j + 1 + tid) * n] = b;
            } else if (tid < C + R) {
                const int a = tid - C;
                int s = rs0 + 1 + a;
                if (s >= RW) s -= RW;
                const double v = W[(size_t)cs0 * RW + s];
                sL[a] = v;
                M[(j + 1 + a) + (long)j * n] = v;
            } else if (tid == C + R) {
                M[j + (long)j * n] = ajj;
            }
        }
        __syncthreads();
        // Rank-1 update of rows j+1..j+R, columns j+1..j+C (pivot-row
        // entries that are zero skipped, as k_lu_band does).
        {
            double l[4];
            int rsl[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int a = lane + 32 * k;
                int s = rs0 + 1 + a;
                if (s >= RW) s -= RW;
                rsl[k] = s;
                l[k] = a < R ? sL[a] : 0.0;
            }
            for (int t = warp; t < C; t += nwarps) {
                const double u = sU[t];
                if (u == 0.0) continue;
                int cs = cs0 + 1 + t;
                if (cs >= CW) cs -= CW;
                double* col = W + (size_t)cs * RW;
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (lane + 32 * k < R) col[rsl[k]] = __dsub_rn(col[rsl[k]], __dmul_rn(l[k], u));
            }
        }
        // The entering row takes row j's slot, the entering column column
        // j's; neither slot is read by this step's update.
        if (has_ent) {
            if (tid < CW) {
                int cs = cs0 + 1 + tid;
                if (cs >= CW) cs -= CW;
                W[(size_t)cs * RW + rs0] = ent;
            } else {
                int s = rs0 + 1 + (tid - CW);
                if (s >= RW) s -= RW;
                W[(size_t)cs0 * RW + s] = ent;
            }
        }
        int rs1 = rs0 + 1, cs1 = cs0 + 1;
        if (rs1 >= RW) rs1 = 0;
        if (cs1 >= CW) cs1 = 0;
        if (warp == 0 && j + 1 < n) {
            // Column j+1 was updated by this warp (t = 0) and its entering
            // entry written by lane 0.
            __syncwarp();
            pivot(j + 1, rs1, cs1);
        }
        rs0 = rs1;
        cs0 = cs1;
        __syncthreads();
    }
    // The interchanges of steps after j applied to column j's multipliers,
    // in step order.
    for (int c = tid; c < n; c += blockDim.x)
        for (int j = c + 1; j < n; j++) {
            const int p = pv[j];
            if (p != j) {
                const double a = M[j + (long)c * n];
                M[j + (long)c * n] = M[p + (long)c * n];
                M[p + (long)c * n] = a;
            }
        }
}

}  // namespace pgmg
