// Device layout of one multigrid level and the index arithmetic shared by
// every kernel.
//
//  * x   (solution, region.hh:50-53): natural order with a one-point zero halo
//        on every side, (m+2)(n+2)(o+2) values; x(i,j,k) at
//        (i+1) + mx*((j+1) + my*(k+1)), mx = m+2, my = n+2.  The halo is never
//        written, so every stencil slot can be read without bounds checks.
//  * r   (source, region.hh:55) and the residual scratch: colour-major,
//        [8][Nc]; colour c = (i&1) | (j&1)<<1 | (k&1)<<2, in-colour index
//        p = ((k>>1)*N2 + (j>>1))*M2 + (i>>1) with M2 = (m+1)/2 etc.
//  * A   (stencils, region.hh:57-59): colour-major structure-of-arrays,
//        [8][27][Nc]: slot q of every point of colour c is contiguous, so a
//        colour sweep streams 27 dense planes.  Slot q = (di+1)+3(dj+1)+9(dk+1);
//        zero outside the point's box (region.hh:252-256).
//  * S   (boxes): natural order, 6 int8 per point, relative [xd,xu,yd,yu,zd,zu];
//        used only during set-up (coarse boxes, parity read-back).
// Nc is M2*N2*O2 rounded up to a multiple of 64, so every plane starts on a
// 256-byte boundary in FP32 and FP64.  Colour sub-grid entries that fall
// outside the grid (odd sizes) hold zero stencils and are never updated.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pgmg {

struct LevelGeom {
    int m, n, o;     // grid size
    int M2, N2, O2;  // colour sub-grid size, (m+1)/2 ...
    long Nc;         // padded points per colour
    long mx, my;     // halo'd x strides: m+2, n+2
    int prd;         // periodic axes: bit 0 x, bit 1 y, bit 2 z
    int pad_;
    long npts;       // m*n*o

    __host__ __device__ inline long xsize() const { return mx * my * (long)(o + 2); }  // halo'd x
    __host__ __device__ inline long xi(int i, int j, int k) const {
        return (i + 1) + mx * ((j + 1) + my * (long)(k + 1));
    }
    __host__ __device__ inline int colour(int i, int j, int k) const {
        return (i & 1) | ((j & 1) << 1) | ((k & 1) << 2);
    }
    __host__ __device__ inline long cidx(int i, int j, int k) const {
        return ((long)(k >> 1) * N2 + (j >> 1)) * M2 + (i >> 1);
    }
    // Index of (i,j,k) in an [8][Nc] array.
    __host__ __device__ inline long ri(int i, int j, int k) const {
        return (long)colour(i, j, k) * Nc + cidx(i, j, k);
    }
    // Index of slot q of (i,j,k) in an [8][27][Nc] array.
    __host__ __device__ inline long ai(int i, int j, int k, int q) const {
        return ((long)colour(i, j, k) * 27 + q) * Nc + cidx(i, j, k);
    }
    __host__ __device__ inline long pi(int i, int j, int k) const {
        return i + (long)m * (j + (long)n * k);
    }
};

// Index decoding with 32-bit unsigned division (index spaces stay below
// 2^32 points for every supported size; 64-bit division costs several times
// more instructions per thread).
__host__ __device__ __forceinline__ void decode_colour(const LevelGeom& g, long p, int& i2, int& j2, int& k2) {
    unsigned u = (unsigned)p, M2 = (unsigned)g.M2, N2 = (unsigned)g.N2;
    unsigned t = u / M2;
    i2 = (int)(u - t * M2);
    k2 = (int)(t / N2);
    j2 = (int)(t - (unsigned)k2 * N2);
}
__host__ __device__ __forceinline__ void decode_nat(const LevelGeom& g, long q, int& i, int& j, int& k) {
    unsigned u = (unsigned)q, m = (unsigned)g.m, n = (unsigned)g.n;
    unsigned t = u / m;
    i = (int)(u - t * m);
    k = (int)(t / n);
    j = (int)(t - (unsigned)k * n);
}

inline LevelGeom make_geom(int m, int n, int o, int prd = 0) {
    LevelGeom g;
    g.m = m; g.n = n; g.o = o;
    g.prd = prd;
    g.M2 = (m + 1) / 2; g.N2 = (n + 1) / 2; g.O2 = (o + 1) / 2;
    long nc = (long)g.M2 * g.N2 * g.O2;
    g.Nc = (nc + 63) / 64 * 64;
    g.mx = m + 2; g.my = n + 2;
    g.pad_ = 0;
    g.npts = (long)m * n * o;
    return g;
}

// Order of the colours in a forward pass of the 8-colour sweep: the four
// colours with i+j+k even first (000, 011, 101, 110 as (i&1, j&1, k&1)),
// then the four odd ones (111, 100, 010, 001); a backward pass takes them in
// reverse.  Any order is a Gauss-Seidel sweep (the points of one colour are
// independent for a 27-point box); this one reduces the residual per
// V-cycle by as much as the reference's lexicographic order also where the
// coefficients vary by four orders of magnitude, where the order 0..7 falls
// 13 % short (129^3, kappa = exp(2.3 g)).  Sequence position s -> colour.
__host__ __device__ __forceinline__ int colour_seq(int s) {
    return (int)((0x42173560u >> (4 * s)) & 7u);
}

// Slab blocking of the 8-colour sweep: a level whose solution array exceeds
// `budget` bytes is swept in `slabs` z-slabs, all 8 colours of slab s before
// slab s+1 (every ordering of point updates is a Gauss-Seidel sweep; within
// a slab and colour the points stay independent).  Slab s covers colour
// sub-grid planes k2 in [O2*s/slabs, O2*(s+1)/slabs).  The rule depends only
// on the level size, the element size and the budget, so the oracle can
// reproduce the same order.
__host__ __device__ inline int slab_count(const LevelGeom& g, int elem_bytes, long long budget) {
    long long bytes = (long long)g.xsize() * elem_bytes;
    if (budget <= 0 || bytes <= budget) return 1;
    long long s = (bytes + budget - 1) / budget;
    return (int)(s < g.O2 ? s : g.O2);
}
__host__ __device__ inline int slab_lo(const LevelGeom& g, int s, int slabs) {
    return (int)((long long)g.O2 * s / slabs);
}

// Per-axis transfer geometry between a fine axis of size ma and its coarse
// axis (ma+2)>>1 (region.cc:14), as rt_scan_grid/slice/row walk it on one
// process (region.cc:665-746): cubes C = 0..last; the lower point 2C always
// exists; the upper point 2C+1 exists unless C is the last cube of an odd
// axis; on an even axis the last cube's upper point (ma-1) "snaps" onto
// coarse C+1 with weight 1 (mask bits 4/32/256).
// An even periodic axis (p, even ma; coarse size ma/2, region.cc:14) has
// cubes C = -1..ma/2-1, all with both points and none snapped: cube -1 is
// the image of cube ma/2-1, whose upper point ma-1 sits just below fine
// point 0 and also transfers to coarse 0.  Indices of such images are
// unwrapped here and wrapped only to address memory (wrap()).
// An odd periodic axis (coarse size (ma+1)/2) transfers like an odd
// non-periodic one: coarse (ma-1)/2 sits on fine ma-1, the next coarse point
// across the seam is coarse 0 on fine ma = 0, and no fine point lies between
// them (igrid_map's odd periodic branch, region.cc:1236-1243); only the
// stencils wrap around.
__host__ __device__ inline bool even_prd(int ma, bool p) { return p && !(ma & 1); }
__host__ __device__ inline int cube_first(int ma, bool p) { return even_prd(ma, p) ? -1 : 0; }
__host__ __device__ inline int cube_last(int ma, bool p = false) {
    if (even_prd(ma, p)) return (ma >> 1) - 1;
    int sm = (ma + 2) >> 1;
    return (ma & 1) ? sm - 1 : sm - 2;
}
__host__ __device__ inline bool has_upper(int C, int ma, bool p = false) { return even_prd(ma, p) || 2 * C + 1 < ma; }
__host__ __device__ inline bool snapped(int C, int ma, bool p = false) { return !p && !(ma & 1) && C == cube_last(ma); }
// One axis of a coarse point whose transfer is the interior one: both cubes
// I-1 and I exist, have their upper point and are not snapped, so the fine
// points 2I-1, 2I, 2I+1 transfer with weights 1/2, 1, 1/2.
__host__ __device__ inline bool inner_axis(int I, int ma) {
    return I >= 1 && I <= cube_last(ma) && has_upper(I, ma) && !snapped(I, ma);
}
// The coarse points of a level split into the interior box -- inner_axis on
// every axis (non-periodic levels only), I in [1, ih], J in [1, jh], K in
// [1, kh] -- and the shell around it.  Kernels that gather per coarse point
// (restriction, Galerkin fill) enumerate the interior first and the shell
// after it, so that the boundary points' general sums (loops with a dozen
// conditions per contribution) run in warps of their own instead of stalling
// the interior warps that hold one of them (every row of coarse points starts
// and ends with one; at 81 points per row, two warps in three did).
struct CoarseSplit {
    int ih, jh, kh;  // last interior index per axis (0: none)
    long n_in;       // interior points
};
__host__ __device__ inline int split_inner_last(int mc, int ma) {
    int last = 0;
    for (int I = 1; I < mc; I++) {
        if (!inner_axis(I, ma)) break;
        last = I;
    }
    return last;
}
__host__ __device__ inline CoarseSplit coarse_split(const LevelGeom& gf, const LevelGeom& gc) {
    CoarseSplit s{0, 0, 0, 0};
    if (gf.prd) return s;  // periodic: no interior box, natural order
    s.ih = split_inner_last(gc.m, gf.m);
    s.jh = split_inner_last(gc.n, gf.n);
    s.kh = split_inner_last(gc.o, gf.o);
    s.n_in = (long)s.ih * s.jh * s.kh;
    return s;
}
// Index t of the non-interior values of an axis whose interior is [1, h]:
// 0, then h+1, h+2, ... (t itself when h = 0).
__host__ __device__ inline int split_shell_index(int t, int h) { return h == 0 ? t : (t == 0 ? 0 : h + t); }
// Coarse point q (0 <= q < gc.npts) in the split order; true if interior.
// The shell: K outside the interior (all I, J); then K inside and J outside
// (all I); then J, K inside and I outside.
__host__ __device__ inline bool split_point(const LevelGeom& gc, const CoarseSplit& sp, long q, int& I, int& J,
                                            int& K) {
    if (q < sp.n_in) {
        const long t = q / sp.ih;
        I = 1 + (int)(q - t * sp.ih);
        J = 1 + (int)(t % sp.jh);
        K = 1 + (int)(t / sp.jh);
        return true;
    }
    q -= sp.n_in;
    const long M = gc.m, N = gc.n, nk = gc.o - sp.kh, nj = N - sp.jh, ni = M - sp.ih;
    if (q < M * N * nk) {
        I = (int)(q % M);
        J = (int)((q / M) % N);
        K = split_shell_index((int)(q / (M * N)), sp.kh);
    } else if ((q -= M * N * nk) < M * nj * sp.kh) {
        I = (int)(q % M);
        J = split_shell_index((int)((q / M) % nj), sp.jh);
        K = 1 + (int)(q / (M * nj));
    } else {
        q -= M * nj * sp.kh;
        I = split_shell_index((int)(q % ni), sp.ih);
        J = 1 + (int)((q / ni) % sp.jh);
        K = 1 + (int)(q / (ni * sp.jh));
    }
    return false;
}

__host__ __device__ inline int wrap(int v, int size, bool p) {
    return p ? (v < 0 ? v + size : (v >= size ? v - size : v)) : v;
}
__host__ __device__ inline bool px(const LevelGeom& g) { return g.prd & 1; }
__host__ __device__ inline bool py(const LevelGeom& g) { return (g.prd >> 1) & 1; }
__host__ __device__ inline bool pz(const LevelGeom& g) { return (g.prd >> 2) & 1; }

// Weight of fine role d (0 lower, 1 upper) of cube C onto coarse index I,
// 0 if the fine point does not transfer to I.
__host__ __device__ inline double tweight(int C, int d, int I, bool snap) {
    if (!d) return C == I ? 1.0 : 0.0;
    if (snap) return C + 1 == I ? 1.0 : 0.0;
    return (C == I || C + 1 == I) ? 0.5 : 0.0;
}

// grid_map (region.cc:1201-1217): a fine global box bound to the coarse one.
__host__ __device__ inline void grid_map(int& lo, int& hi, int ma, bool p = false) {
    if (p) {
        lo = lo < 0 ? (lo - ((ma & 1) ? 2 : 1)) / 2 : lo >> 1;
        hi = (hi + (((ma & 1) && hi > ma) ? 3 : 2)) >> 1;
        return;
    }
    lo = (!(ma & 1) && lo == ma - 1 ? lo + 1 : lo) >> 1;
    hi = (hi + 2) >> 1;
}

// igrid_map with the crop to the stencil box (region.cc:1231-1259): the fine
// range a coarse index gathers from, and its coincident fine index.  On an
// even periodic axis coarse i <-> fine 2i with range [2i-1, 2i+2); on an odd
// one the coarse images i < 0 and i >= (ma+1)/2 sit one fine point closer
// (the short cell at the seam) and ranges end at the seam.
__host__ __device__ inline int igrid_map(int& lo, int& hi, int blo, int bhi, int i, int ma, bool p = false) {
    int j = i * 2;
    if (p && (ma & 1)) {
        int llo, hhi;
        if (j < 0) { j += 1; llo = -ma; hhi = 0; }
        else if (j >= ma) { j -= 1; llo = ma; hhi = 2 * ma; }
        else { llo = 0; hhi = ma; }
        lo = j == llo ? llo : j - 1;
        hi = j == hhi - 1 ? hhi : j + 2;
    }
    else if (p) { lo = j - 1; hi = j + 2; }
    else if (ma & 1) { lo = j == 0 ? 0 : j - 1; hi = j == ma - 1 ? ma : j + 2; }
    else if (j == ma) { lo = ma - 1; hi = ma; j = ma - 1; }
    else { lo = j == 0 ? 0 : j - 1; hi = j == ma - 2 ? ma - 1 : j + 2; }
    if (lo < blo) lo = blo;
    if (hi > bhi) hi = bhi;
    return j;
}

// Periodic images in the one-point halo of x: halo index -1 holds the value
// of size-1 and halo index size that of 0, on periodic axes only (the halo of
// a non-periodic axis stays zero).  Writes v at (i,j,k)'s images.
template <class T>
__device__ __forceinline__ void store_images(const LevelGeom& g, T* x, int i, int j, int k, T v) {
    int ia = (g.prd & 1) ? (i == 0 ? g.m : (i == g.m - 1 ? -1 : -2)) : -2;
    int ja = (g.prd & 2) ? (j == 0 ? g.n : (j == g.n - 1 ? -1 : -2)) : -2;
    int ka = (g.prd & 4) ? (k == 0 ? g.o : (k == g.o - 1 ? -1 : -2)) : -2;
    if (ia == -2 && ja == -2 && ka == -2) return;
    for (int s = 1; s < 8; s++) {
        int ii = (s & 1) ? ia : i, jj = (s & 2) ? ja : j, kk = (s & 4) ? ka : k;
        if (ii == -2 || jj == -2 || kk == -2) continue;
        x[g.xi(ii, jj, kk)] = v;
    }
}

// Arithmetic helpers: EXACT = round every product and sum separately, as the
// reference's x86-64 build does (no fused multiply-add), so results match it
// bit for bit; otherwise fused multiply-add.
template <class T> __device__ inline T mul_rn(T a, T b);
template <> __device__ inline double mul_rn<double>(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ inline float mul_rn<float>(float a, float b) { return __fmul_rn(a, b); }
template <class T> __device__ inline T add_rn(T a, T b);
template <> __device__ inline double add_rn<double>(double a, double b) { return __dadd_rn(a, b); }
template <> __device__ inline float add_rn<float>(float a, float b) { return __fadd_rn(a, b); }
template <class T> __device__ inline T sub_rn(T a, T b);
template <> __device__ inline double sub_rn<double>(double a, double b) { return __dsub_rn(a, b); }
template <> __device__ inline float sub_rn<float>(float a, float b) { return __fsub_rn(a, b); }

template <bool EXACT, class T> __device__ inline T madd(T acc, T a, T b) {
    if (EXACT) return add_rn<T>(acc, mul_rn<T>(a, b));
    return fma(a, b, acc);
}

// L2 eviction-priority hints.  Stencil coefficients and sources are
// streamed once per pass (evict_first, and not kept in L1); the solution
// vector is re-read by every colour pass and by the residual, so it is loaded
// and stored with evict_last to keep as much of it in L2 as fits.
__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ double ld_stream(const double* a, uint64_t pol) {
    double v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_stream(const float* a, uint64_t pol) {
    float v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
    return v;
}
// 128-bit streaming loads of 2 doubles / 4 floats (16-byte aligned).
__device__ __forceinline__ void ld_stream_v(const double* a, uint64_t pol, double (&v)[2]) {
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
        : "=d"(v[0]), "=d"(v[1]) : "l"(a), "l"(pol));
}
// 64-bit streaming loads of 2 floats (8-byte aligned).
__device__ __forceinline__ void ld_stream_v(const float* a, uint64_t pol, float (&v)[2]) {
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
        : "=f"(v[0]), "=f"(v[1]) : "l"(a), "l"(pol));
}
__device__ __forceinline__ void ld_stream_v(const float* a, uint64_t pol, float (&v)[4]) {
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
        : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]) : "l"(a), "l"(pol));
}
__device__ __forceinline__ double ld_keep(const double* a, uint64_t pol) {
    double v;
    asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_keep(const float* a, uint64_t pol) {
    float v;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ void st_keep(double* a, double v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(a), "d"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_keep(float* a, float v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(a), "f"(v), "l"(pol) : "memory");
}

// Programmatic dependent launch.  A kernel launched with the programmatic
// stream-serialization attribute may be scheduled while the kernel before it
// in the stream is still draining; it must not touch global memory before
// pdl_wait() returns (every prerequisite grid complete, its writes visible).
// pdl_trigger() lets the next such kernel be scheduled.  Both do nothing in a
// kernel launched without the attribute.  Every kernel of the V-cycle and of
// the solve loops starts with both calls.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_enter() {
    pdl_wait();
    pdl_trigger();
}

// Offset of slot q in the halo'd x array.
__host__ __device__ inline long slot_off(const LevelGeom& g, int q) {
    int di = q % 3 - 1, dj = (q / 3) % 3 - 1, dk = q / 9 - 1;
    return di + g.mx * (dj + g.my * dk);
}

}  // namespace pgmg
