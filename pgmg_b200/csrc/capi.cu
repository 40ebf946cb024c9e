// C ABI of the B200 multigrid library: handle and device arena, hierarchy
// plan, operator set-up, the V-cycle engine and the solves.  See
// include/pgmg_dev.h for the contract of every entry point.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

#include "../../include/pgmg_dev.h"
#include "handle.cuh"

using namespace pgmg;

namespace {

pgmg_status fail(pgmg_handle* h, pgmg_status st, const char* fmt, ...) {
    if (h) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(h->err, sizeof(h->err), fmt, ap);
        va_end(ap);
    }
    return st;
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(h, PGMG_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)
#define CKL()             \
    do {                  \
        h->launches++;    \
        CK(cudaGetLastError()); \
    } while (0)
// A V-cycle or solve-loop kernel (one that starts with pdl_enter()).
#define LAUNCH(grid, block, ...)                                              \
    do {                                                                      \
        h->launches++;                                                        \
        CK(launch_k(h->stream, h->pdl, grid, block, __VA_ARGS__));            \
    } while (0)
#define TRY(expr)                          \
    do {                                   \
        pgmg_status s_ = (expr);           \
        if (s_ != PGMG_OK) return s_;      \
    } while (0)

// Hierarchy plan (multigrid::setup_hierarchy, multigrid.cc:17-85; coarse
// sizes region.cc:14: (m+2)>>1, or (m+1)>>1 on a periodic axis).
int plan_levels(const pgmg_dims& d, LevelGeom* g) {
    int nl = 0;
    int m = d.m, n = d.n, o = d.o;
    int prd = (d.x_prd ? 1 : 0) | (d.y_prd ? 2 : 0) | (d.z_prd ? 4 : 0);
    g[nl++] = make_geom(m, n, o, prd);
    while ((long)m * n * o > 1024 && nl < kMaxLevels) {
        m = (m + (d.x_prd ? 1 : 2)) >> 1; n = (n + (d.y_prd ? 1 : 2)) >> 1; o = (o + (d.z_prd ? 1 : 2)) >> 1;
        g[nl++] = make_geom(m, n, o, prd);
    }
    return nl;
}

// Lays out every buffer in the arena (or only counts bytes if base is null).
void carve(pgmg_handle* h) {
    Arena& a = h->arena;
    a.used = 0;
    bool mixed = h->dims.precision == PGMG_MIXED;
    long maxblocks = 0;
    for (int l = 0; l < h->nl; l++) {
        Level& L = h->L[l];
        const LevelGeom& g = L.g;
        L.A64 = a.take<double>(8 * 27 * g.Nc);
        L.x64 = a.take<double>(g.xsize());
        L.r64 = a.take<double>(8 * g.Nc);
        L.res64 = a.take<double>(8 * g.Nc);
        L.S = a.take<int8_t>(6 * g.npts);
        if (mixed) {
            L.A32 = a.take<float>(8 * 27 * g.Nc);
            L.x32 = a.take<float>(g.xsize());
            L.r32 = a.take<float>(8 * g.Nc);
            L.res32 = a.take<float>(8 * g.Nc);
        }
        long b = nblk((long)g.M2 * g.N2 * g.O2) * 8;
        if (b > maxblocks) maxblocks = b;
    }
    long n = h->L[h->nl - 1].g.npts;
    h->nex = n;
    if (n < kMaxExact) {
        h->M = a.take<double>(n * n);
        h->Minv = a.take<double>(n * n);
        h->lubuf = a.take<double>(n);
        h->piv = a.take<int>(n);
    }
    h->info = a.take<int>(4);
    h->bar = a.take<GridBar>(1);
    h->plan64 = a.take<CoarsePlan<double>>(1);
    h->plan32 = a.take<CoarsePlan<float>>(1);
    h->partials = a.take<double>(2 * maxblocks);
    h->norm_dev = a.take<double>(2);
    const LevelGeom& g0 = h->L[0].g;
    size_t coef_all = (size_t)27 * g0.npts;
    size_t cap = (size_t)64 << 20;  // 512 MB of doubles
    size_t st = coef_all < cap ? coef_all : cap;
    if (st < (size_t)g0.npts) st = g0.npts;
    if (st < (size_t)27 * g0.m * g0.n) st = (size_t)27 * g0.m * g0.n;
    h->stage_elems = st;
    h->stage = a.take<double>(st);
}

pgmg_status check_level(pgmg_handle* h, int level) {
    if (!h) return PGMG_ERR_ARG;
    if (level < 0 || level >= h->nl) return fail(h, PGMG_ERR_ARG, "level %d out of range [0,%d)", level, h->nl);
    return PGMG_OK;
}

// ---------------------------------------------------------------------------
// V-cycle engine, templated on the storage type.

template <class T> View<T> view(Level& L);
template <> View<double> view<double>(Level& L) { return view64(L); }
template <> View<float> view<float>(Level& L) { return view32(L); }

// Periodic images of a level's solution (no-op on non-periodic levels).
template <class T>
pgmg_status wrap_level(pgmg_handle* h, int l) {
    const LevelGeom& g = h->L[l].g;
    if (!g.prd) return PGMG_OK;
    LAUNCH(nblk(halo_cells(g)), kBlock, k_halo_wrap<T>, g, view<T>(h->L[l]).x);
    return PGMG_OK;
}

// All sweeps of one leg on level l in one cooperative launch (k_sweeps_grid).
template <class T>
pgmg_status grid_sweeps(pgmg_handle* h, int l, int mode, int sweeps, unsigned extra = 0) {
    Level& L = h->L[l];
    View<T> v = view<T>(L);
    const LevelGeom& g = L.g;
    long nc = (long)g.M2 * g.N2 * g.O2;
    long need = nblk(nc, 512);
    int cap = h->grid_blocks[std::is_same<T, float>::value ? 1 : 0];
    int blocks = (int)(need < cap ? need : cap);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks, 1, 1);
    cfg.blockDim = dim3(512, 1, 1);
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    h->launches++;
    CK(cudaLaunchKernelEx(&cfg, k_sweeps_grid<T>, g, v.x, (const T*)v.r, (const T*)v.A, sweeps, mode, h->bar,
                          (unsigned)blocks + extra));
    return PGMG_OK;
}

// A bounded device wait that ran out -- a grid barrier of the persistent
// sweeps or an mbarrier wait of the TMA colour pass (reported once, then
// cleared).
pgmg_status check_grid(pgmg_handle* h) {
    if (!h->grid_max && !h->gs_tma) return PGMG_OK;
    int e[2] = {0, 0};
    CK(cudaMemcpyAsync(e, &h->bar->err, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (!e[0] && !e[1]) return PGMG_OK;
    CK(cudaMemsetAsync(h->bar, 0, sizeof(GridBar), h->stream));
    if (e[0]) return fail(h, PGMG_ERR_TIMEOUT, "a grid barrier of the persistent sweep kernel ran out of time");
    return fail(h, PGMG_ERR_TIMEOUT, "an mbarrier wait of the TMA colour pass ran out of time");
}

// Threads per block of level l's colour sweep (PGMG_OPT_GS_BLOCK, or the
// level's own PGMG_OPT_GS_BLOCK_LEVELS entry).
int sweep_block(const pgmg_handle* h, int l) {
    if (l < 1 || l > 15) return h->gs_block;
    const int code = (int)((h->gs_block_lv >> (2 * (l - 1))) & 3);
    return code == 0 ? h->gs_block : code == 1 ? 128 : code == 2 ? 256 : 512;
}

// One colour pass of k_gs_colour_tma (128 threads per CTA when the sweep
// block is 128, else 256).
template <class T>
pgmg_status gs_tma_pass(pgmg_handle* h, const LevelGeom& g, View<T>& v, int col, int rev, long nc, unsigned extra) {
    h->launches++;
    if (h->gs_block == 128) {
        CK(launch_k_smem(h->stream, h->pdl, dim3((unsigned)nblk(nc, 128)), dim3(128), gs_tma_smem<T, 128>(),
                         k_gs_colour_tma<T, 128>, g, v.x, (const T*)v.r, (const T*)v.A, col, rev, &h->bar->tma_err,
                         extra));
    } else {
        CK(launch_k_smem(h->stream, h->pdl, dim3((unsigned)nblk(nc, 256)), dim3(256), gs_tma_smem<T, 256>(),
                         k_gs_colour_tma<T, 256>, g, v.x, (const T*)v.r, (const T*)v.A, col, rev, &h->bar->tma_err,
                         extra));
    }
    return PGMG_OK;
}

template <class T>
pgmg_status gs_level(pgmg_handle* h, int l, int mode, int smoother, int sweeps = 1) {
    Level& L = h->L[l];
    View<T> v = view<T>(L);
    const LevelGeom& g = L.g;
    const int bs = sweep_block(h, l);
    // An odd periodic axis (possible on the bottom level only) has no valid
    // 8-colouring: sweep that level lexicographically.
    if (g.prd && ((px(g) && (g.m & 1)) || (py(g) && (g.n & 1)) || (pz(g) && (g.o & 1))))
        smoother = PGMG_SMOOTH_LEX;
    if (smoother == PGMG_SMOOTH_LEX && g.prd) {
        // region::gauss_seidel (region.cc:355-361, 456-457) refreshes the
        // ghosts before the forward and before the backward pass and sweeps
        // with them fixed: the images are refreshed before each pass (and
        // after the last), and the hyperplane kernel reads but never writes
        // them.
        int np = num_planes(g);
        for (int s = 0; s < sweeps; s++) {
            for (int pass = 0; pass < (mode ? 2 : 1); pass++) {
                TRY(wrap_level<T>(h, l));
                for (int tt = 0; tt < np; tt++) {
                    int t = pass ? np - 1 - tt : tt;
                    Plane P = plane_range(g, t);
                    long nw = (long)(P.kmax - P.kmin + 1) * P.jw;
                    if (nw <= 0) continue;
                    LAUNCH(nblk(nw), kBlock, k_gs_plane<T>, g, v.x, v.r, v.A, t, P);
                }
            }
        }
        return wrap_level<T>(h, l);
    }
    if (smoother == PGMG_SMOOTH_LEX) {
        if (g.npts <= kLexBlockMax) {
            LAUNCH(1, 1024, k_gs_lex_block<T>, g, v.x, v.r, v.A, sweeps, mode);
            return PGMG_OK;
        }
        int np = num_planes(g);
        for (int s = 0; s < sweeps; s++)
            for (int pass = 0; pass < (mode ? 2 : 1); pass++)
                for (int tt = 0; tt < np; tt++) {
                    int t = pass ? np - 1 - tt : tt;
                    Plane P = plane_range(g, t);
                    long nw = (long)(P.kmax - P.kmin + 1) * P.jw;
                    if (nw <= 0) continue;
                    LAUNCH(nblk(nw), kBlock, k_gs_plane<T>, g, v.x, v.r, v.A, t, P);
                }
        return PGMG_OK;
    }
    if (g.npts <= kMc8BlockMax && !g.prd) {
        LAUNCH(1, 1024, k_gs_mc8_block<T>, g, v.x, v.r, v.A, sweeps, mode, h->slab_budget);
        return PGMG_OK;
    }
    int S = slab_count(g, (int)sizeof(T), h->slab_budget);
    if (S == 1 && !g.prd && h->gs_tma > 0 && g.npts <= h->gs_tma) {
        // Stencils and sources staged by bulk copies (k_gs_colour_tma).
        long nc = (long)g.M2 * g.N2 * g.O2;
        for (int s = 0; s < sweeps; s++)
            for (int pass = 0; pass < (mode ? 2 : 1); pass++)
                for (int cc = 0; cc < 8; cc++) {
                    int col = colour_seq(pass ? 7 - cc : cc);
                    int rev = h->gs_alt ? (cc & 1) : 0;
                    TRY(gs_tma_pass<T>(h, g, v, col, rev, nc, 0u));
                }
        return PGMG_OK;
    }
    if (S == 1 && !g.prd && g.npts <= h->grid_max && sweeps > 0 &&
        h->grid_blocks[std::is_same<T, float>::value ? 1 : 0] > 0)
        return grid_sweeps<T>(h, l, mode, sweeps);
    if (S == 1 && !g.prd && g.npts <= h->gs_prefetch) {
        // Stencil loaded before the launch dependency (k_gs_colour_pf); on
        // levels of at most gs_l2pf points each pass also prefetches the
        // next pass's stencils into L2.
        long nc = (long)g.M2 * g.N2 * g.O2;
        const int per = mode ? 16 : 8, total = sweeps * per;
        const bool l2pf = g.npts <= h->gs_l2pf;
        for (int st = 0; st < total; st++) {
            int cc = st % per;
            int col = colour_seq(cc < 8 ? cc : 15 - cc);
            int nx = st + 1 < total && l2pf ? colour_seq((st + 1) % per < 8 ? (st + 1) % per : 15 - (st + 1) % per) : -1;
            int rev = h->gs_alt ? (cc & 1) : 0;
            if (bs == 128)
                LAUNCH(nblk(nc, 128), 128, k_gs_colour_pf<T, 128>, g, v.x, v.r, v.A, col, rev, nx);
            else if (bs == 512)
                LAUNCH(nblk(nc, 512), 512, k_gs_colour_pf<T, 512>, g, v.x, v.r, v.A, col, rev, nx);
            else
                LAUNCH(nblk(nc, 256), 256, k_gs_colour_pf<T, 256>, g, v.x, v.r, v.A, col, rev, nx);
        }
        return PGMG_OK;
    }
    if (S == 1 && !g.prd && h->gs_vec) {
        // Vector loads, V colour points per thread: 16-byte vectors
        // (gs_vec 1), or 2 points per thread (gs_vec 2: 8-byte vectors of
        // FP32; for FP64 the same as 1).  On the levels the variants above
        // do not take (with the default thresholds, level 0 of a large grid).
        constexpr int V16 = 16 / sizeof(T);
        const int V = h->gs_vec == 2 ? 2 : V16;
        long nthr = ((long)g.M2 * g.N2 * g.O2 + V - 1) / V;
        for (int s = 0; s < sweeps; s++)
            for (int pass = 0; pass < (mode ? 2 : 1); pass++)
                for (int cc = 0; cc < 8; cc++) {
                    int col = colour_seq(pass ? 7 - cc : cc);
                    int rev = h->gs_alt ? (cc & 1) : 0;
                    if (V == V16) {
                        if (bs == 128)
                            LAUNCH(nblk(nthr, 128), 128, k_gs_colour_v<T, 128>, g, v.x, v.r, v.A, col, rev);
                        else if (bs == 512)
                            LAUNCH(nblk(nthr, 512), 512, k_gs_colour_v<T, 512>, g, v.x, v.r, v.A, col, rev);
                        else
                            LAUNCH(nblk(nthr, 256), 256, k_gs_colour_v<T, 256>, g, v.x, v.r, v.A, col, rev);
                    } else {
                        if (bs == 128)
                            LAUNCH(nblk(nthr, 128), 128, k_gs_colour_v<T, 128, 2>, g, v.x, v.r, v.A, col, rev);
                        else if (bs == 512)
                            LAUNCH(nblk(nthr, 512), 512, k_gs_colour_v<T, 512, 2>, g, v.x, v.r, v.A, col, rev);
                        else
                            LAUNCH(nblk(nthr, 256), 256, k_gs_colour_v<T, 256, 2>, g, v.x, v.r, v.A, col, rev);
                    }
                }
        return PGMG_OK;
    }
    for (int s = 0; s < sweeps; s++)
        for (int pass = 0; pass < (mode ? 2 : 1); pass++)
            for (int ss = 0; ss < S; ss++) {
                int sl = pass ? S - 1 - ss : ss;
                int k2lo = slab_lo(g, sl, S), k2hi = slab_lo(g, sl + 1, S);
                long np = (long)(k2hi - k2lo) * g.M2 * g.N2;
                for (int cc = 0; cc < 8; cc++) {
                    int col = colour_seq(pass ? 7 - cc : cc);
                    int rev = h->gs_alt ? (cc & 1) : 0;  // alternate the traversal direction
                    if (g.prd)
                        LAUNCH(nblk(np), kBlock, k_gs_colour<T, true, true>, g, v.x, v.r, v.A, col, k2lo, k2hi, rev);
                    else if (bs == 128)
                        LAUNCH(nblk(np, 128), 128, k_gs_colour<T, true, false, 128>, g, v.x, v.r, v.A, col, k2lo,
                               k2hi, rev);
                    else if (bs == 512)
                        LAUNCH(nblk(np, 512), 512, k_gs_colour<T, true, false, 512>, g, v.x, v.r, v.A, col, k2lo,
                               k2hi, rev);
                    else
                        LAUNCH(nblk(np), kBlock, k_gs_colour<T, true>, g, v.x, v.r, v.A, col, k2lo, k2hi, rev);
                }
            }
    return PGMG_OK;
}

template <class T>
pgmg_status residual_level(pgmg_handle* h, int l, T* out, double* partials) {
    Level& L = h->L[l];
    View<T> v = view<T>(L);
    const LevelGeom& g = L.g;
    dim3 grid((unsigned)(8 * nblk((long)g.M2 * g.N2 * g.O2)));  // colours interleaved
    LAUNCH(grid, kBlock, k_residual<T, T, true>, g, v.x, v.r, v.A, out, partials);
    return PGMG_OK;
}

template <class T, class Tile>
pgmg_status fused_restrict(pgmg_handle* h, Level& F, Level& Cl, View<T>& vf, View<T>& vc) {
    const LevelGeom& gc = Cl.g;
    dim3 grid((unsigned)((gc.m + Tile::tx - 1) / Tile::tx), (unsigned)((gc.n + Tile::ty - 1) / Tile::ty),
              (unsigned)((gc.o + Tile::kc - 1) / Tile::kc));
    const size_t sm = Tile::template smem<T>();  // limit set in prepare_device_kernels
    h->launches++;
    CK(launch_k_smem(h->stream, h->pdl, grid, dim3(Tile::threads), sm, k_resrestrict<T, Tile>, F.g, gc,
                     (const T*)vf.x, (const T*)vf.r, (const T*)vf.A, vc.r, vc.x));
    return PGMG_OK;
}

template <class T>
pgmg_status restrict_level(pgmg_handle* h, int l) {
    Level& F = h->L[l - 1];
    Level& Cl = h->L[l];
    View<T> vf = view<T>(F), vc = view<T>(Cl);
    if (!F.g.prd && h->fused_restrict) return fused_restrict<T, RrSmall>(h, F, Cl, vf, vc);
    TRY(residual_level<T>(h, l - 1, vf.res, nullptr));
    if (F.g.prd)
        LAUNCH(nblk(Cl.g.npts), kBlock, k_restrict<T, true>, F.g, Cl.g, vf.res, vc.r, vc.x);
    else
        LAUNCH(nblk(Cl.g.npts), kBlock, k_restrict_fast<T>, F.g, Cl.g, coarse_split(F.g, Cl.g), vf.res, vc.r, vc.x);
    return wrap_level<T>(h, l);
}

template <class T>
pgmg_status interp_level(pgmg_handle* h, int l) {
    Level& F = h->L[l - 1];
    Level& Cl = h->L[l];
    LAUNCH(nblk((long)F.g.M2 * F.g.N2 * F.g.O2), kBlock, k_interp_cube<T>, F.g, Cl.g, view<T>(F).x, view<T>(Cl).x);
    return wrap_level<T>(h, l - 1);
}

template <class T>
pgmg_status coarse_solve_t(pgmg_handle* h, int smoother) {
    int lb = h->nl - 1;
    Level& L = h->L[lb];
    View<T> v = view<T>(L);
    if (h->lu_ok) {
        if (h->dims.coarse == PGMG_COARSE_LU_EXACT) {
            LAUNCH(1, 1024, k_lu_solve_exact<T>, L.g, h->M, h->piv, v.r, v.x, h->lubuf);
        } else {
            long thr = L.g.npts * 32;
            LAUNCH(nblk(thr), kBlock, k_lu_apply<T>, L.g, h->Minv, v.r, v.x);
        }
        return wrap_level<T>(h, lb);
    }
    // region::solve_exact fallback: pgmg_gs_exact plain (mode 0) sweeps of
    // the cycle's smoother (region_tr.cc:557; the reference's own smoother is
    // the lexicographic one).
    return gs_level<T>(h, lb, 0, smoother, kGsExact);
}

// Fills the coarse-cycle plan of a handle (host copy).
template <class T>
void fill_plan(pgmg_handle* h, int first, CoarsePlan<T>& P) {
    P.first = first;
    P.nl = h->nl;
    P.lu_ok = h->lu_ok;
    P.slab_budget = h->slab_budget;
    P.v_down = h->v_down;
    P.v_up = h->v_up;
    P.Minv = h->Minv;
    for (int l = 0; l < h->nl; l++) {
        View<T> v = view<T>(h->L[l]);
        P.g[l] = h->L[l].g;
        P.A[l] = v.A; P.x[l] = v.x; P.r[l] = v.r; P.res[l] = v.res;
    }
}

// Refreshes the device copies of the plans (after set-up and option changes).
pgmg_status upload_plans(pgmg_handle* h) {
    CoarsePlan<double> p64;
    fill_plan<double>(h, h->coarse_first, p64);
    CK(cudaMemcpyAsync(h->plan64, &p64, sizeof(p64), cudaMemcpyHostToDevice, h->stream));
    if (h->dims.precision == PGMG_MIXED) {
        CoarsePlan<float> p32;
        fill_plan<float>(h, h->coarse_first, p32);
        CK(cudaMemcpyAsync(h->plan32, &p32, sizeof(p32), cudaMemcpyHostToDevice, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    return PGMG_OK;
}

template <class T> const CoarsePlan<T>* plan_of(pgmg_handle* h);
template <> const CoarsePlan<double>* plan_of<double>(pgmg_handle* h) { return h->plan64; }
template <> const CoarsePlan<float>* plan_of<float>(pgmg_handle* h) { return h->plan32; }

template <class T>
pgmg_status launch_coarse(pgmg_handle* h, int first, int mode) {
    (void)first;  // the device plan carries h->coarse_first
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(h->cluster_size, 1, 1);
    cfg.blockDim = dim3(kClusterThreads, 1, 1);
    cfg.stream = h->stream;
    if (h->coarse_shared) {
        // Room for the largest x copy of a level the cluster sweeps (levels
        // whose copy does not fit sweep from global memory).
        long need = 0;
        for (int l = h->coarse_first; l < h->nl; l++) {
            const LevelGeom& g = h->L[l].g;
            // The x copy and the staged stencils, for levels where both fit;
            // else the level's z-plane windows (c_sweeps_window), where
            // every CTA's points fit in one pass of its threads.
            long b = shared_copy(g, h->cluster_size).bytes((int)sizeof(T));
            long nc = (long)g.M2 * g.N2 * g.O2;
            if (b > kCoarseXsMax && (nc + h->cluster_size - 1) / h->cluster_size <= kClusterThreads)
                b = window_bytes(g, h->cluster_size, (int)sizeof(T));
            if (b <= kCoarseXsMax && b > need) need = b;
        }
        cfg.dynamicSmemBytes = (size_t)need;
    }
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = h->cluster_size;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = h->pdl ? 2 : 1;
    const int* no_map = nullptr;
    const int* no_flags = nullptr;
    CK(cudaLaunchKernelEx(&cfg, k_coarse_cycle<T>, plan_of<T>(h), no_map, no_flags, mode));
    h->launches++;
    return PGMG_OK;
}

// Clusters of `size` CTAs of the coarse cycle that fit on the device at once (0: not launchable).
template <class T>
int probe_cluster(int size) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(size, 1, 1);
    cfg.blockDim = dim3(kClusterThreads, 1, 1);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = size;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (size > 8 && cudaFuncSetAttribute(k_coarse_cycle<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_coarse_cycle<T>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// One V-cycle (multigrid::v_cycle, multigrid.cc:88-106).  With the 8-colour
// smoother the levels from h->coarse_first down run as one cluster kernel;
// the LU-exact coarse solve and the lexicographic smoother use the grid
// kernels on every level.
template <class T>
pgmg_status vcycle_t(pgmg_handle* h, int mode, int smoother) {
    int ml = h->nl;
    bool cl = smoother == PGMG_SMOOTH_MC8 && h->cluster_size > 0 && h->dims.coarse != PGMG_COARSE_LU_EXACT;
    int lc = cl ? h->coarse_first : ml;
    int top = lc < ml ? lc : ml - 1;
    for (int i = 0; i < top; i++) {
        TRY(gs_level<T>(h, i, mode, smoother, h->v_down + i));
        TRY(restrict_level<T>(h, i + 1));
    }
    if (lc < ml) TRY(launch_coarse<T>(h, lc, mode));
    else TRY(coarse_solve_t<T>(h, smoother));
    for (int i = top; i > 0; i--) {
        TRY(interp_level<T>(h, i));
        TRY(gs_level<T>(h, i - 1, mode, smoother, h->v_up + i - 1));
    }
    return PGMG_OK;
}

// vcycle_t with an event recorded after each stage (ev[0] before the first);
// returns the number of events recorded into ev, and the coarse level.
template <class T>
pgmg_status vcycle_profiled(pgmg_handle* h, int smoother, std::vector<cudaEvent_t>& ev, std::vector<int>& tag,
                            int* lc_out) {
    int ml = h->nl;
    bool cl = smoother == PGMG_SMOOTH_MC8 && h->cluster_size > 0 && h->dims.coarse != PGMG_COARSE_LU_EXACT;
    int lc = cl ? h->coarse_first : ml;
    int top = lc < ml ? lc : ml - 1;
    *lc_out = top;
    auto mark = [&](int t) -> pgmg_status {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        ev.push_back(e);
        tag.push_back(t);
        CK(cudaEventRecord(e, h->stream));
        return PGMG_OK;
    };
    TRY(mark(-1));
    for (int i = 0; i < top; i++) {
        TRY(gs_level<T>(h, i, 0, smoother, h->v_down + i));
        TRY(mark(4 * i + 0));
        TRY(restrict_level<T>(h, i + 1));
        TRY(mark(4 * i + 1));
    }
    if (lc < ml) TRY(launch_coarse<T>(h, lc, 0));
    else TRY(coarse_solve_t<T>(h, smoother));
    TRY(mark(4 * kMaxLevels));
    for (int i = top; i > 0; i--) {
        TRY(interp_level<T>(h, i));
        TRY(mark(4 * (i - 1) + 2));
        TRY(gs_level<T>(h, i - 1, 0, smoother, h->v_up + i - 1));
        TRY(mark(4 * (i - 1) + 3));
    }
    return PGMG_OK;
}

void drop_graphs(pgmg_handle* h) {
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++)
            for (int c = 0; c < 2; c++)
                if (h->vgraph[a][b][c]) {
                    cudaGraphExecDestroy(h->vgraph[a][b][c]);
                    h->vgraph[a][b][c] = nullptr;
                }
}

// One V-cycle as a CUDA graph: the launch sequence of vcycle_t is captured
// once per (precision, mode, smoother) and replayed, so the several hundred
// small launches of the coarse levels cost no host launch overhead.
template <class T>
pgmg_status run_vcycle(pgmg_handle* h, int mode, int smoother) {
    TraceRange tr(std::is_same<T, float>::value ? "pgmg V-cycle fp32" : "pgmg V-cycle fp64");
    if (!h->use_graphs) return vcycle_t<T>(h, mode, smoother);
    int a = std::is_same<T, float>::value ? 1 : 0, b = mode ? 1 : 0, c = smoother == PGMG_SMOOTH_LEX ? 1 : 0;
    cudaGraphExec_t& ex = h->vgraph[a][b][c];
    if (!ex) {
        long long before = h->launches;
        CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        pgmg_status st = vcycle_t<T>(h, mode, smoother);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
        if (st != PGMG_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        CK(e);
        e = cudaGraphInstantiate(&ex, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            ex = nullptr;
            return fail(h, PGMG_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
        }
        h->vgraph_nodes[a][b][c] = h->launches - before;
        h->launches = before;
    }
    CK(cudaGraphLaunch(ex, h->stream));
    h->launches += h->vgraph_nodes[a][b][c];
    return PGMG_OK;
}

// A residual check's norms: call check_begin before launching the kernel
// that writes the partial sums, then reduce_and_read, which leaves the two
// norms in h->norm_host.  With the pinned pair the reduction writes them to
// host memory directly, and the host waits in two steps: a blocking wait on
// the event recorded before the residual kernel (the thread wakes while that
// kernel still runs), then polling of the event after the reduction -- so
// the norms are read within microseconds of being written, not a thread
// wake-up later.
constexpr long kNormPolls = 1L << 20;  // then a blocking wait

pgmg_status check_begin(pgmg_handle* h) {
    if (h->norm_pin) CK(cudaEventRecord(h->ev_pre, h->stream));
    return PGMG_OK;
}

// The reduction of a check, enqueued; read_norms waits for it.  Work
// enqueued between the two runs while the host waits.
pgmg_status reduce_launch(pgmg_handle* h, long nb) {
    if (!h->norm_pin) {
        LAUNCH(1, 1024, k_reduce_partials, h->partials, nb, h->norm_dev);
        CK(cudaMemcpyAsync(h->norm_host, h->norm_dev, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        return PGMG_OK;
    }
    LAUNCH(1, 1024, k_reduce_partials, h->partials, nb, h->norm_pin);
    CK(cudaEventRecord(h->ev_post, h->stream));
    return PGMG_OK;
}

pgmg_status read_norms(pgmg_handle* h) {
    if (!h->norm_pin) {
        CK(cudaStreamSynchronize(h->stream));
        return PGMG_OK;
    }
    CK(cudaEventSynchronize(h->ev_pre));
    cudaError_t e = cudaErrorNotReady;
    for (long i = 0; i < kNormPolls && e == cudaErrorNotReady; i++) e = cudaEventQuery(h->ev_post);
    if (e == cudaErrorNotReady) e = cudaEventSynchronize(h->ev_post);
    CK(e);
    h->norm_host[0] = h->norm_pin[0];
    h->norm_host[1] = h->norm_pin[1];
    return PGMG_OK;
}

pgmg_status reduce_and_read(pgmg_handle* h, long nb) {
    TRY(reduce_launch(h, nb));
    return read_norms(h);
}

// Norms of a level (FP64 data) into h->norm_host; synchronises.
pgmg_status norms64(pgmg_handle* h, int l, double* res2, double* rhs2) {
    Level& L = h->L[l];
    TRY(check_begin(h));
    TRY(residual_level<double>(h, l, nullptr, h->partials));
    TRY(reduce_and_read(h, nblk((long)L.g.M2 * L.g.N2 * L.g.O2) * 8));
    if (res2) *res2 = h->norm_host[0];
    if (rhs2) *rhs2 = h->norm_host[1];
    return PGMG_OK;
}

// x64 += x32 on level 0 (the FP64 update of iterative refinement).
pgmg_status add_correction(pgmg_handle* h) {
    Level& L0 = h->L[0];
    const LevelGeom& g = L0.g;
    if (((uintptr_t)L0.x64 | (uintptr_t)L0.x32) & 15) {
        LAUNCH(nblk(g.npts), kBlock, k_add_correction, g, L0.x64, L0.x32);
    } else {
        long n = g.xsize();
        LAUNCH(nblk((n + 3) / 4), kBlock, k_add_correction_flat, L0.x64, L0.x32, n);
    }
    return PGMG_OK;
}

// One step of FP64 iterative refinement around an FP32 V-cycle:
// r32 = b - A64 x64 (FP64 residual, stored FP32, with norms of the current
// x), e32 = V-cycle(r32) from e32 = 0, x64 += e32.
pgmg_status ir_step(pgmg_handle* h, int mode, int smoother, double* res2, double* rhs2) {
    Level& L0 = h->L[0];
    const LevelGeom& g = L0.g;
    dim3 grid((unsigned)(8 * nblk((long)g.M2 * g.N2 * g.O2)));  // colours interleaved
    if (res2 || rhs2) TRY(check_begin(h));
    LAUNCH(grid, kBlock, k_residual<double, float, true>, g, L0.x64, L0.r64, L0.A64, L0.r32,
           (res2 || rhs2) ? h->partials : nullptr);
    long nb = nblk((long)g.M2 * g.N2 * g.O2) * 8;
    if (res2 || rhs2) {
        TRY(reduce_and_read(h, nb));
        if (res2) *res2 = h->norm_host[0];
        if (rhs2) *rhs2 = h->norm_host[1];
    }
    CK(cudaMemsetAsync(L0.x32, 0, g.xsize() * sizeof(float), h->stream));  // e = 0 (halo too)
    TRY(wrap_level<float>(h, 0));
    TRY(run_vcycle<float>(h, mode, smoother));
    TRY(add_correction(h));
    TRY(wrap_level<double>(h, 0));
    return PGMG_OK;
}

pgmg_status lu_setup(pgmg_handle* h) {
    TraceRange tr("pgmg coarse LU");
    h->lu_ok = 0;
    int lb = h->nl - 1;
    Level& L = h->L[lb];
    long n = L.g.npts;
    if (n >= kMaxExact || h->dims.coarse == PGMG_COARSE_GS) return PGMG_OK;
    CK(cudaMemsetAsync(h->M, 0, sizeof(double) * n * n, h->stream));
    CK(cudaMemsetAsync(h->info, 0, sizeof(int) * 4, h->stream));
    k_lu_build<<<nblk(n), kBlock, 0, h->stream>>>(L.g, L.A64, L.S, h->M);
    CKL();
    {
        // Bandwidth of the 27-point stencil in natural order (a periodic
        // axis couples the first and last planes: no band).
        int kb = L.g.prd ? (int)n - 1 : 1 + L.g.m + L.g.m * L.g.n;
        if (kb > (int)n - 1) kb = (int)n - 1;
        size_t wsm = lu_window_smem((int)n, kb, kb);
        if (h->lu_window && !L.g.prd && wsm <= kLuWindowSmemMax && kb <= 128) {
            // The active band window in shared memory (same factors; the
            // limit is set in prepare_device_kernels; a lane updates at most
            // 4 rows, so kl <= 128).
            k_lu_window<<<1, 1024, wsm, h->stream>>>(h->M, (int)n, kb, kb, h->piv, h->info);
        } else {
            k_lu_band<<<1, 1024, 0, h->stream>>>(h->M, (int)n, kb, kb, h->piv, h->info);
        }
        CKL();
    }
    k_lu_extent<<<nblk(n * 32), kBlock, 0, h->stream>>>(h->M, (int)n, h->info + 1);
    CKL();
    int info4[4] = {0, 0, 0, 0};
    double u0 = 0, un = 0;
    CK(cudaMemcpyAsync(info4, h->info, sizeof(info4), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(&u0, h->M, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(&un, h->M + n * n - 1, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const int info = info4[0], bl = info4[1], bu = info4[2];
    // Conditioning check of region_tr.cc:524-533.
    double hi = fabs(u0), lo = fabs(un);
    if (info != 0 || hi == 0 || lo / hi < 2.220446049250313e-16 * 1e4) return PGMG_OK;
    if (h->dims.coarse == PGMG_COARSE_LU) {
        const unsigned nbk = (unsigned)((n + kInvWarps - 1) / kInvWarps);
        const size_t ism = kInvWarps * n * sizeof(double);
        if (h->lu_inv_band && bl <= 128 && bu <= 256) {
            k_lu_inverse_band<4, 8><<<nbk, 32 * kInvWarps, ism, h->stream>>>(h->M, h->piv, (int)n, bl, bu, h->Minv);
        } else if (h->lu_inv_band && bl <= 256 && bu <= 256) {
            k_lu_inverse_band<8, 4><<<nbk, 32 * kInvWarps, ism, h->stream>>>(h->M, h->piv, (int)n, bl, bu, h->Minv);
        } else {
            k_lu_inverse<<<(unsigned)n, 256, n * sizeof(double), h->stream>>>(h->M, h->piv, (int)n, h->Minv);
        }
        CKL();
    }
    h->lu_ok = 1;
    return PGMG_OK;
}

void guide_update(pgmg_handle* h, int extras) {
    int diter = -1 + h->period * extras;
    if (h->use_avg) {
        double di = h->iter - h->iter_avg;
        int zscore = (int)(di / sqrt(h->iter_var));
        if (zscore > 0) diter -= zscore;
        h->iter_avg = (1 - h->alpha) * h->iter_avg + h->alpha * h->iter;
        h->iter_var = (1 - h->alpha) * (h->iter_var + h->alpha * di * di);
    }
    h->iter += diter;
    if (h->iter < h->period) h->iter = 2 * h->period - 1;
}

// Once per device, before the first handle on it does any work: the
// dynamic shared-memory limits of the kernels that need more than 48 KiB,
// and a query of every set-up kernel's attributes, which also loads it.
// With lazy module loading a kernel is otherwise loaded at its first use,
// and a first use on one thread (a server's set-up thread) while another
// thread captures a CUDA graph invalidates that capture.
pgmg_status prepare_device_kernels(int device) {
    static std::mutex mu;
    static bool done[64] = {};
    std::lock_guard<std::mutex> lk(mu);
    if (device < 0 || device >= 64) return PGMG_ERR_ARG;
    if (done[device]) return PGMG_OK;
    bool ok = true;
    ok = ok && cudaFuncSetAttribute(k_lu_window, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLuWindowSmemMax) ==
                   cudaSuccess;
    ok = ok && cudaFuncSetAttribute(k_rat_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRtSmem) == cudaSuccess;
    ok = ok && cudaFuncSetAttribute(k_rat_fill, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRatSmem) == cudaSuccess;
    ok = ok && cudaFuncSetAttribute(k_lu_inverse_band<4, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(kInvWarps * kMaxExact * sizeof(double))) == cudaSuccess;
    ok = ok && cudaFuncSetAttribute(k_lu_inverse_band<8, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(kInvWarps * kMaxExact * sizeof(double))) == cudaSuccess;
    ok = ok && cudaFuncSetAttribute(k_gs_colour_tma<double, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)gs_tma_smem<double, 256>()) == cudaSuccess;
    ok = ok && cudaFuncSetAttribute(k_gs_colour_tma<float, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)gs_tma_smem<float, 256>()) == cudaSuccess;
    cudaFuncAttributes fa;
    const void* setup_kernels[] = {(const void*)k_gs_colour_tma<double, 128>, (const void*)k_gs_colour_tma<float, 128>,(const void*)k_lu_build,       (const void*)k_lu_band,
                                   (const void*)k_lu_inverse,     (const void*)k_lu_inverse_band<4, 8>,
                                   (const void*)k_lu_inverse_band<8, 4>,
                                   (const void*)k_lu_extent,      (const void*)k_rat_bounds,
                                   (const void*)k_rat_fill,       (const void*)k_rat_fill_small,
                                   (const void*)k_assemble_q1,    (const void*)k_rhs_uniform,
                                   (const void*)k_cell_exp,
                                   (const void*)k_resrestrict<double, RrSmall>,
                                   (const void*)k_resrestrict<float, RrSmall>};
    for (const void* k : setup_kernels) ok = ok && cudaFuncGetAttributes(&fa, k) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        return PGMG_ERR_CUDA;
    }
    done[device] = true;
    return PGMG_OK;
}

bool is_device_ptr(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

// ===========================================================================
extern "C" {

pgmg_status pgmg_dev_plan_bytes(const pgmg_dims* dims, size_t* bytes) {
    if (!dims || !bytes) return PGMG_ERR_ARG;
    if (dims->m < 2 || dims->n < 2 || dims->o < 2) return PGMG_ERR_ARG;
    pgmg_handle tmp;
    tmp.dims = *dims;
    LevelGeom g[kMaxLevels];
    tmp.nl = plan_levels(*dims, g);
    for (int l = 0; l < tmp.nl; l++) tmp.L[l].g = g[l];
    carve(&tmp);
    *bytes = tmp.arena.used;
    return PGMG_OK;
}

// Page-locked host pairs for the handles' residual norms (the reduction
// kernel writes each check's two sums straight into its handle's pair).  They
// come from blocks of kPinPairs pairs that are allocated once, portable to
// every device, and reused for the life of the process, so that creating and
// destroying a handle -- which a server does for every new request -- does
// not page-lock memory: that allocation is slow, and CUDA lets it serialise
// the work of concurrent streams.
constexpr int kPinPairs = 256;
// (The list is never destroyed, so a handle destroyed during process exit,
// after static destructors have run, can still return its pair.)
static std::mutex g_pin_mu;
static std::vector<double*>& g_pin_free = *new std::vector<double*>;

static double* pin_pair_take() {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    if (g_pin_free.empty()) {
        void* block = nullptr;
        if (cudaHostAlloc(&block, kPinPairs * 2 * sizeof(double), cudaHostAllocPortable | cudaHostAllocMapped) !=
            cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        for (int i = kPinPairs - 1; i >= 0; i--) g_pin_free.push_back(static_cast<double*>(block) + 2 * i);
    }
    double* p = g_pin_free.back();
    g_pin_free.pop_back();
    return p;
}

static void pin_pair_give(double* p) {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pin_free.push_back(p);
}

static pgmg_status create_common(const pgmg_dims* dims, void* mem, size_t mem_bytes, pgmg_handle** out) {
    if (!dims || !out) return PGMG_ERR_ARG;
    *out = nullptr;
    if (dims->m < 2 || dims->n < 2 || dims->o < 2) return PGMG_ERR_ARG;
    if (dims->precision != PGMG_FP64 && dims->precision != PGMG_MIXED) return PGMG_ERR_ARG;
    if (dims->coarse < PGMG_COARSE_LU || dims->coarse > PGMG_COARSE_LU_EXACT) return PGMG_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return PGMG_ERR_NO_DEVICE;
    }
    pgmg_handle* h = new pgmg_handle;
    h->dims = *dims;
    if (dims->device >= 0) {
        if (dims->device >= ndev) { delete h; return PGMG_ERR_ARG; }
        cudaSetDevice(dims->device);
    }
    cudaGetDevice(&h->device);
    if (prepare_device_kernels(h->device) != PGMG_OK) {
        delete h;
        return PGMG_ERR_CUDA;
    }
    LevelGeom g[kMaxLevels];
    h->nl = plan_levels(*dims, g);
    for (int l = 0; l < h->nl; l++) h->L[l].g = g[l];
    h->prd = g[0].prd;
    // Periodic axes of odd size (on any level) are supported: their
    // transfers follow igrid_map's odd periodic branch, and a level with one
    // is swept lexicographically (no 8-colouring separates the neighbours
    // across its seam, which have equal parity).
    carve(h);  // count
    size_t bytes = h->arena.used;
    if (mem) {
        if (mem_bytes < bytes || (reinterpret_cast<uintptr_t>(mem) & 255)) {
            delete h;
            return PGMG_ERR_MEMORY;
        }
        h->arena.base = static_cast<char*>(mem);
        h->own_arena = false;
    } else {
        cudaError_t e = cudaMalloc(&h->arena.base, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            delete h;
            return PGMG_ERR_MEMORY;
        }
    }
    h->arena.size = bytes;
    carve(h);  // assign
    if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        pgmg_dev_destroy(h);
        return PGMG_ERR_CUDA;
    }
    h->stream = h->own;
    h->norm_pin = pin_pair_take();
    if (!h->norm_pin || cudaEventCreateWithFlags(&h->ev_pre, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_post, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (h->norm_pin) pin_pair_give(h->norm_pin);
        h->norm_pin = nullptr;  // checks fall back to a copy and a stream synchronisation
    }
    for (int size : {16, 8}) {
        if (probe_cluster<double>(size) > 0 && probe_cluster<float>(size) > 0) {
            h->cluster_size = size;
            break;
        }
    }
    if (cudaFuncSetAttribute(k_coarse_cycle<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, kCoarseXsMax) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_coarse_cycle<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, kCoarseXsMax) !=
            cudaSuccess) {
        cudaGetLastError();
        h->coarse_shared = false;
    }
    h->coarse_first = h->nl - 1;
    for (int l = 0; l < h->nl; l++)
        if (h->L[l].g.npts <= kClusterMax) { h->coarse_first = l; break; }
    {
        int dev_sms = 0, nb64 = 0, nb32 = 0;
        cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, h->device);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb64, k_sweeps_grid<double>, 512, 0) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb32, k_sweeps_grid<float>, 512, 0) != cudaSuccess) {
            cudaGetLastError();
            nb64 = nb32 = 0;
        }
        h->grid_blocks[0] = nb64 * dev_sms;
        h->grid_blocks[1] = nb32 * dev_sms;
    }
    if (h->prd) {
        // Periodic levels keep their halo images current between kernels
        // (k_halo_wrap), so they run with the per-level kernels only.
        h->cluster_size = 0;
        h->coarse_first = h->nl;
    }
    if (cudaMemsetAsync(h->arena.base, 0, bytes, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
        pgmg_dev_destroy(h);
        return PGMG_ERR_CUDA;
    }
    *out = h;
    return PGMG_OK;
}

pgmg_status pgmg_dev_create(const pgmg_dims* dims, pgmg_handle** out) { return create_common(dims, nullptr, 0, out); }

pgmg_status pgmg_dev_create_in(const pgmg_dims* dims, void* mem, size_t bytes, pgmg_handle** out) {
    if (!mem) return PGMG_ERR_ARG;
    return create_common(dims, mem, bytes, out);
}

pgmg_status pgmg_dev_destroy(pgmg_handle* h) {
    if (!h) return PGMG_ERR_ARG;
    if (h->stream) cudaStreamSynchronize(h->stream);
    drop_graphs(h);
    if (h->norm_pin) pin_pair_give(h->norm_pin);
    if (h->ev_pre) cudaEventDestroy(h->ev_pre);
    if (h->ev_post) cudaEventDestroy(h->ev_post);
    if (h->ostream) cudaStreamSynchronize(h->ostream);
    if (h->ev_out) cudaEventDestroy(h->ev_out);
    if (h->ostream) cudaStreamDestroy(h->ostream);
    if (h->arena.base && h->own_arena) cudaFree(h->arena.base);
    if (h->own) cudaStreamDestroy(h->own);
    delete h;
    return PGMG_OK;
}

pgmg_status pgmg_dev_set_stream(pgmg_handle* h, void* s) {
    if (!h) return PGMG_ERR_ARG;
    h->stream = s ? static_cast<cudaStream_t>(s) : h->own;
    return PGMG_OK;
}

pgmg_status pgmg_dev_sync(pgmg_handle* h) {
    if (!h) return PGMG_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    return check_grid(h);
}

const char* pgmg_dev_last_error(pgmg_handle* h) { return h ? h->err : "null handle"; }

pgmg_status pgmg_dev_launch_count(pgmg_handle* h, long long* n) {
    if (!h || !n) return PGMG_ERR_ARG;
    *n = h->launches;
    return PGMG_OK;
}

pgmg_status pgmg_dev_set_option(pgmg_handle* h, int key, long long value) {
    if (!h) return PGMG_ERR_ARG;
    switch (key) {
        case PGMG_OPT_GRAPHS:
            h->use_graphs = value != 0;
            break;
        case PGMG_OPT_CLUSTER_FIRST:
            if (value < 0 || value > h->nl) return fail(h, PGMG_ERR_ARG, "cluster level %lld out of range", value);
            h->coarse_first = (int)value;
            break;
        case PGMG_OPT_CLUSTER_SIZE:
            if (value != 0 && value != 1 && value != 2 && value != 4 && value != 8 && value != 16)
                return fail(h, PGMG_ERR_ARG, "cluster size must be 0, 1, 2, 4, 8 or 16");
            if (value && h->prd) return fail(h, PGMG_ERR_UNSUPPORTED, "periodic problems run without the cluster coarse cycle");
            if (value && (probe_cluster<double>((int)value) <= 0 || probe_cluster<float>((int)value) <= 0))
                return fail(h, PGMG_ERR_UNSUPPORTED, "cluster of %lld CTAs not launchable", value);
            h->cluster_size = (int)value;
            break;
        case PGMG_OPT_SLAB_BUDGET:
            h->slab_budget = value;
            break;
        case PGMG_OPT_PDL:
            h->pdl = value != 0;
            break;
        case PGMG_OPT_GS_VECTOR:
            if (value < 0 || value > 2) return fail(h, PGMG_ERR_ARG, "gs_vector must be 0, 1 or 2");
            h->gs_vec = (int)value;
            break;
        case PGMG_OPT_GS_ALTERNATE:
            h->gs_alt = value != 0;
            break;
        case PGMG_OPT_COARSE_SHARED:
            h->coarse_shared = value != 0;
            break;
        case PGMG_OPT_FUSED_RESTRICT:
            h->fused_restrict = value != 0;
            break;
        case PGMG_OPT_LU_WINDOW:
            h->lu_window = value != 0;
            break;
        case PGMG_OPT_LU_INVERSE_BAND:
            h->lu_inv_band = value != 0;
            break;
        case PGMG_OPT_GS_BLOCK_LEVELS:
            if (value < 0 || value >= (1LL << 30)) return fail(h, PGMG_ERR_ARG, "gs_block_levels: 2 bits per level 1..15");
            h->gs_block_lv = value;
            break;
        case PGMG_OPT_GS_TMA:
            if (value < 0) return fail(h, PGMG_ERR_ARG, "gs_tma must be >= 0");
            h->gs_tma = value;
            break;
        case PGMG_OPT_RAT_TILE:
            h->rat_tile = value != 0;
            break;
        case PGMG_OPT_GS_L2_PREFETCH:
            if (value < 0) return fail(h, PGMG_ERR_ARG, "gs_l2_prefetch must be >= 0");
            h->gs_l2pf = value;
            break;
        case PGMG_OPT_GS_PREFETCH:
            if (value < 0) return fail(h, PGMG_ERR_ARG, "gs_prefetch must be >= 0");
            h->gs_prefetch = value;
            break;
        case PGMG_OPT_INNER_DIGITS:
            if (value < 1 || value > 7) return fail(h, PGMG_ERR_ARG, "inner reduction digits must be 1..7");
            h->inner_digits = (int)value;
            break;
        case PGMG_OPT_GRID_MAX:
            if (value < 0) return fail(h, PGMG_ERR_ARG, "grid_max must be >= 0");
            if (value && (h->grid_blocks[0] == 0 || h->grid_blocks[1] == 0))
                return fail(h, PGMG_ERR_UNSUPPORTED, "persistent sweep kernel not launchable");
            h->grid_max = value;
            break;
        case PGMG_OPT_GS_BLOCK:
            if (value != 128 && value != 256 && value != 512)
                return fail(h, PGMG_ERR_ARG, "colour-sweep block must be 128, 256 or 512 threads");
            h->gs_block = (int)value;
            break;
        case PGMG_OPT_V_DOWN:
        case PGMG_OPT_V_UP:
        case PGMG_OPT_V_BOTTOM:
            if (value < 0 || value > 1000) return fail(h, PGMG_ERR_ARG, "sweep count %lld out of range", value);
            (key == PGMG_OPT_V_DOWN ? h->v_down : key == PGMG_OPT_V_UP ? h->v_up : h->v_bottom) = (int)value;
            break;
        default:
            return fail(h, PGMG_ERR_ARG, "unknown option %d", key);
    }
    drop_graphs(h);
    if (h->built) TRY(upload_plans(h));
    return PGMG_OK;
}

pgmg_status pgmg_dev_get_option(pgmg_handle* h, int key, long long* value) {
    if (!h || !value) return PGMG_ERR_ARG;
    switch (key) {
        case PGMG_OPT_GRAPHS: *value = h->use_graphs; return PGMG_OK;
        case PGMG_OPT_CLUSTER_FIRST: *value = h->coarse_first; return PGMG_OK;
        case PGMG_OPT_CLUSTER_SIZE: *value = h->cluster_size; return PGMG_OK;
        case PGMG_OPT_SLAB_BUDGET: *value = h->slab_budget; return PGMG_OK;
        case PGMG_OPT_V_DOWN: *value = h->v_down; return PGMG_OK;
        case PGMG_OPT_V_UP: *value = h->v_up; return PGMG_OK;
        case PGMG_OPT_V_BOTTOM: *value = h->v_bottom; return PGMG_OK;
        case PGMG_OPT_PDL: *value = h->pdl; return PGMG_OK;
        case PGMG_OPT_GS_BLOCK: *value = h->gs_block; return PGMG_OK;
        case PGMG_OPT_GRID_MAX: *value = h->grid_max; return PGMG_OK;
        case PGMG_OPT_GS_VECTOR: *value = h->gs_vec; return PGMG_OK;
        case PGMG_OPT_INNER_DIGITS: *value = h->inner_digits; return PGMG_OK;
        case PGMG_OPT_GS_ALTERNATE: *value = h->gs_alt; return PGMG_OK;
        case PGMG_OPT_GS_PREFETCH: *value = h->gs_prefetch; return PGMG_OK;
        case PGMG_OPT_COARSE_SHARED: *value = h->coarse_shared; return PGMG_OK;
        case PGMG_OPT_FUSED_RESTRICT: *value = h->fused_restrict; return PGMG_OK;
        case PGMG_OPT_LU_WINDOW: *value = h->lu_window; return PGMG_OK;
        case PGMG_OPT_LU_INVERSE_BAND: *value = h->lu_inv_band; return PGMG_OK;
        case PGMG_OPT_GS_BLOCK_LEVELS: *value = h->gs_block_lv; return PGMG_OK;
        case PGMG_OPT_GS_TMA: *value = h->gs_tma; return PGMG_OK;
        case PGMG_OPT_RAT_TILE: *value = h->rat_tile; return PGMG_OK;
        case PGMG_OPT_GS_L2_PREFETCH: *value = h->gs_l2pf; return PGMG_OK;
    }
    return fail(h, PGMG_ERR_ARG, "unknown option %d", key);
}

pgmg_status pgmg_dev_set_smoother(pgmg_handle* h, int smoother) {
    if (!h || (smoother != PGMG_SMOOTH_MC8 && smoother != PGMG_SMOOTH_LEX)) return PGMG_ERR_ARG;
    h->dims.smoother = smoother;
    return PGMG_OK;
}

pgmg_status pgmg_dev_num_levels(pgmg_handle* h, int* nl) {
    if (!h || !nl) return PGMG_ERR_ARG;
    *nl = h->nl;
    return PGMG_OK;
}

pgmg_status pgmg_dev_level_dims(pgmg_handle* h, int level, int* mno) {
    TRY(check_level(h, level));
    if (!mno) return PGMG_ERR_ARG;
    mno[0] = h->L[level].g.m; mno[1] = h->L[level].g.n; mno[2] = h->L[level].g.o;
    return PGMG_OK;
}

pgmg_status pgmg_dev_memory(pgmg_handle* h, size_t* bytes) {
    if (!h || !bytes) return PGMG_ERR_ARG;
    *bytes = h->arena.size;
    return PGMG_OK;
}

pgmg_status pgmg_dev_upload_level0(pgmg_handle* h, const double* coef27, const int* S6) {
    if (!h || !coef27) return PGMG_ERR_ARG;
    TraceRange tr("pgmg upload_level0");
    Level& L = h->L[0];
    const LevelGeom& g = L.g;
    // Boxes: validate on the host (region.hh:498-506 reads them per point).
    std::vector<int8_t> s8(6 * g.npts);
    if (S6) {
        std::vector<int> tmp;
        const int* sp = S6;
        if (is_device_ptr(S6)) {
            tmp.resize(6 * g.npts);
            CK(cudaMemcpy(tmp.data(), S6, sizeof(int) * 6 * g.npts, cudaMemcpyDeviceToHost));
            sp = tmp.data();
        }
        for (long p = 0; p < g.npts; p++) {
            int i = (int)(p % g.m), j = (int)((p / g.m) % g.n), k = (int)(p / ((long)g.m * g.n));
            const int* b = sp + 6 * p;
            int c[3] = {i, j, k}, ext[3] = {g.m, g.n, g.o};
            for (int a = 0; a < 3; a++) {
                int lo = b[2 * a], hi = b[2 * a + 1];
                if (lo < -1 || hi > 2 || lo >= hi || lo > 0 || hi < 1)
                    return fail(h, PGMG_ERR_ARG, "box of point (%d,%d,%d) axis %d is [%d,%d): must contain 0 and lie in [-1,2)", i, j, k, a, lo, hi);
                if (!((h->prd >> a) & 1) && (c[a] + lo < 0 || c[a] + hi > ext[a]))
                    return fail(h, PGMG_ERR_ARG, "box of point (%d,%d,%d) leaves the non-periodic grid on axis %d", i, j, k, a);
                s8[6 * p + 2 * a] = (int8_t)lo;
                s8[6 * p + 2 * a + 1] = (int8_t)hi;
            }
        }
    } else {
        for (long p = 0; p < g.npts; p++) {
            int i = (int)(p % g.m), j = (int)((p / g.m) % g.n), k = (int)(p / ((long)g.m * g.n));
            int c[3] = {i, j, k}, ext[3] = {g.m, g.n, g.o};
            for (int a = 0; a < 3; a++) {
                bool pa = (h->prd >> a) & 1;
                s8[6 * p + 2 * a] = (int8_t)(pa || c[a] > 0 ? -1 : 0);
                s8[6 * p + 2 * a + 1] = (int8_t)(pa || c[a] < ext[a] - 1 ? 2 : 1);
            }
        }
    }
    CK(cudaMemcpyAsync(L.S, s8.data(), s8.size(), cudaMemcpyHostToDevice, h->stream));
    // Stencils, chunked by z-planes through the staging buffer.
    long plane = 27L * g.m * g.n;
    int kchunk = (int)(h->stage_elems / plane);
    if (kchunk < 1) return fail(h, PGMG_ERR_INTERNAL, "staging buffer smaller than one plane");
    for (int k0 = 0; k0 < g.o; k0 += kchunk) {
        int k1 = k0 + kchunk < g.o ? k0 + kchunk : g.o;
        size_t cnt = (size_t)plane * (k1 - k0);
        CK(cudaMemcpyAsync(h->stage, coef27 + (size_t)plane * k0, cnt * sizeof(double), cudaMemcpyDefault, h->stream));
        k_coef_to_cm<double><<<nblk((long)cnt), kBlock, 0, h->stream>>>(g, k0, k1, h->stage, L.S, L.A64);
        CKL();
    }
    CK(cudaStreamSynchronize(h->stream));  // s8 and the caller's array are released on return
    h->uploaded = true;
    h->built = false;
    return PGMG_OK;
}

pgmg_status pgmg_dev_assemble_q1(pgmg_handle* h, const double* cells, int from_log, double sigma) {
    if (!h) return PGMG_ERR_ARG;
    TraceRange tr("pgmg assemble_q1");
    if (h->prd) return fail(h, PGMG_ERR_UNSUPPORTED, "the Q1 generator builds Dirichlet problems only");
    Level& L = h->L[0];
    const LevelGeom& g = L.g;
    const double* dc = nullptr;
    if (cells) {
        size_t nc = (size_t)(g.m - 1) * (g.n - 1) * (g.o - 1);
        if (is_device_ptr(cells)) dc = cells;
        else {
            CK(cudaMemcpyAsync(h->stage, cells, nc * sizeof(double), cudaMemcpyHostToDevice, h->stream));
            dc = h->stage;
        }
    }
    if (dc && from_log) {
        // kappa of every cell once, into the level's residual scratch (free
        // during set-up; at least npts > cells doubles).
        size_t nc = (size_t)(g.m - 1) * (g.n - 1) * (g.o - 1);
        k_cell_exp<<<nblk((long)nc), kBlock, 0, h->stream>>>(dc, (long)nc, sigma, L.res64);
        CKL();
        dc = L.res64;
        from_log = 0;
    }
    int mx = g.m > g.n ? (g.m > g.o ? g.m : g.o) : (g.n > g.o ? g.n : g.o);
    double hh = 1.0 / (double)(mx - 1);
    k_assemble_q1<<<nblk(g.npts, 128), 128, 0, h->stream>>>(g, dc, from_log, sigma, hh, L.A64, L.S);
    CKL();
    CK(cudaStreamSynchronize(h->stream));
    h->uploaded = true;
    h->built = false;
    return PGMG_OK;
}

pgmg_status pgmg_dev_rhs_uniform(pgmg_handle* h, uint64_t seed) {
    if (!h) return PGMG_ERR_ARG;
    Level& L = h->L[0];
    k_rhs_uniform<<<nblk(L.g.npts), 256, 0, h->stream>>>(L.g, seed, L.r64);
    CKL();
    return PGMG_OK;
}

pgmg_status pgmg_dev_build_rat(pgmg_handle* h) {
    if (!h) return PGMG_ERR_ARG;
    TraceRange tr("pgmg build_rat");
    if (!h->uploaded) return fail(h, PGMG_ERR_SETUP, "level-0 stencils not uploaded");
    drop_graphs(h);
    for (int l = 1; l < h->nl; l++) {
        Level& F = h->L[l - 1];
        Level& Cl = h->L[l];
        k_rat_bounds<<<nblk(Cl.g.npts), kBlock, 0, h->stream>>>(F.g, Cl.g, F.S, Cl.S);
        CKL();
        if (Cl.g.npts <= kRatSmallMax) {
            k_rat_fill_small<<<nblk(Cl.g.npts * 32, kRatSmallBlock), kRatSmallBlock, 0, h->stream>>>(F.g, Cl.g, F.A64,
                                                                                                   F.S, Cl.A64);
        } else if (!F.g.prd && h->rat_tile) {
            dim3 grid((unsigned)((Cl.g.m + kRtX - 1) / kRtX), (unsigned)Cl.g.n, (unsigned)((Cl.g.o + kRtKC - 1) / kRtKC));
            k_rat_tile<<<grid, kRtThreads, kRtSmem, h->stream>>>(F.g, Cl.g, F.A64, F.S, Cl.A64);
        } else {
            k_rat_fill<<<nblk(Cl.g.npts, kRatBlock), kRatBlock, kRatSmem, h->stream>>>(F.g, Cl.g, coarse_split(F.g, Cl.g),
                                                                                      F.A64, F.S, Cl.A64);
        }
        CKL();
    }
    if (h->dims.precision == PGMG_MIXED)
        for (int l = 0; l < h->nl; l++) {
            long cnt = 8L * 27 * h->L[l].g.Nc;
            k_cast<double, float><<<nblk(cnt), kBlock, 0, h->stream>>>(h->L[l].A64, h->L[l].A32, cnt);
            CKL();
        }
    TRY(lu_setup(h));
    CK(cudaStreamSynchronize(h->stream));
    TRY(upload_plans(h));
    h->built = true;
    return PGMG_OK;
}

pgmg_status pgmg_dev_lu_enabled(pgmg_handle* h, int* enabled) {
    if (!h || !enabled) return PGMG_ERR_ARG;
    *enabled = h->lu_ok;
    return PGMG_OK;
}

pgmg_status pgmg_dev_get_coef(pgmg_handle* h, int level, double* coef27) {
    TRY(check_level(h, level));
    if (!coef27) return PGMG_ERR_ARG;
    Level& L = h->L[level];
    const LevelGeom& g = L.g;
    // Chunked by z-planes through the staging buffer.
    long plane = 27L * g.m * g.n;
    int kchunk = (int)(h->stage_elems / plane);
    if (kchunk < 1) return fail(h, PGMG_ERR_INTERNAL, "staging buffer smaller than one plane");
    for (int k0 = 0; k0 < g.o; k0 += kchunk) {
        int k1 = k0 + kchunk < g.o ? k0 + kchunk : g.o;
        size_t cnt = (size_t)plane * (k1 - k0);
        k_cm_to_coef<double><<<nblk((long)cnt), kBlock, 0, h->stream>>>(g, k0, k1, L.A64, h->stage);
        CKL();
        CK(cudaMemcpyAsync(coef27 + (size_t)plane * k0, h->stage, cnt * sizeof(double), cudaMemcpyDefault,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));  // the staging buffer is reused by the next chunk
    }
    return PGMG_OK;
}

pgmg_status pgmg_dev_get_boxes(pgmg_handle* h, int level, int* S6) {
    TRY(check_level(h, level));
    if (!S6) return PGMG_ERR_ARG;
    const LevelGeom& g = h->L[level].g;
    std::vector<int8_t> s8(6 * g.npts);
    CK(cudaMemcpyAsync(s8.data(), h->L[level].S, s8.size(), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    std::vector<int> tmp(6 * g.npts);
    for (size_t q = 0; q < s8.size(); q++) tmp[q] = s8[q];
    CK(cudaMemcpy(S6, tmp.data(), sizeof(int) * tmp.size(), cudaMemcpyDefault));
    return PGMG_OK;
}

pgmg_status pgmg_dev_set_field(pgmg_handle* h, int level, int field, const double* src) {
    TRY(check_level(h, level));
    if (field == PGMG_FIELD_X) h->x0_zero = false;
    if (!src || (field != PGMG_FIELD_X && field != PGMG_FIELD_R)) return PGMG_ERR_ARG;
    Level& L = h->L[level];
    const LevelGeom& g = L.g;
    CK(cudaMemcpyAsync(h->stage, src, sizeof(double) * g.npts, cudaMemcpyDefault, h->stream));
    if (field == PGMG_FIELD_X) k_nat_to_x<double><<<nblk(g.npts), kBlock, 0, h->stream>>>(g, h->stage, L.x64);
    else k_nat_to_cm<double><<<nblk(g.npts), kBlock, 0, h->stream>>>(g, h->stage, L.r64);
    CKL();
    if (field == PGMG_FIELD_X) TRY(wrap_level<double>(h, level));
    CK(cudaStreamSynchronize(h->stream));
    return PGMG_OK;
}

pgmg_status pgmg_dev_get_field(pgmg_handle* h, int level, int field, double* dst) {
    TRY(check_level(h, level));
    if (!dst) return PGMG_ERR_ARG;
    Level& L = h->L[level];
    const LevelGeom& g = L.g;
    if (field == PGMG_FIELD_X) k_x_to_nat<double><<<nblk(g.npts), kBlock, 0, h->stream>>>(g, L.x64, h->stage);
    else if (field == PGMG_FIELD_R) k_cm_to_nat<double><<<nblk(g.npts), kBlock, 0, h->stream>>>(g, L.r64, h->stage);
    else if (field == PGMG_FIELD_RES) {
        TRY(residual_level<double>(h, level, L.res64, nullptr));
        k_cm_to_nat<double><<<nblk(g.npts), kBlock, 0, h->stream>>>(g, L.res64, h->stage);
    } else return PGMG_ERR_ARG;
    CKL();
    CK(cudaMemcpyAsync(dst, h->stage, sizeof(double) * g.npts, cudaMemcpyDefault, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return PGMG_OK;
}

pgmg_status pgmg_dev_apply(pgmg_handle* h, int level, const double* in, double* out) {
    TRY(check_level(h, level));
    if (!in || !out) return PGMG_ERR_ARG;
    Level& L = h->L[level];
    const LevelGeom& g = L.g;
    CK(cudaMemcpyAsync(h->stage, in, sizeof(double) * g.npts, cudaMemcpyDefault, h->stream));
    k_apply<double><<<nblk(g.npts), kBlock, 0, h->stream>>>(g, L.A64, h->stage, L.res64);
    CKL();
    CK(cudaMemcpyAsync(out, L.res64, sizeof(double) * g.npts, cudaMemcpyDefault, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return PGMG_OK;
}

}  // extern "C"

namespace {

// One PCG helper reduction (k_helper_partials) over a level, read back.
pgmg_status helper_reduce(pgmg_handle* h, int level, int what, const double* ext, double* out) {
    Level& L = h->L[level];
    const LevelGeom& g = L.g;
    long nb = nblk(g.npts);
    k_helper_partials<<<(unsigned)nb, kBlock, 0, h->stream>>>(g, L.x64, L.r64, L.A64, ext, what, h->partials);
    CKL();
    if (what == 2) k_reduce_max<<<1, 1024, 0, h->stream>>>(h->partials, nb, h->norm_dev);
    else k_reduce_partials<<<1, 1024, 0, h->stream>>>(h->partials, nb, h->norm_dev);
    CKL();
    double v[2] = {0, 0};
    CK(cudaMemcpyAsync(v, h->norm_dev, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *out = v[0];
    return PGMG_OK;
}

}  // namespace

extern "C" {

pgmg_status pgmg_dev_source_soln_dot(pgmg_handle* h, int level, double* out) {
    TRY(check_level(h, level));
    if (!out) return PGMG_ERR_ARG;
    return helper_reduce(h, level, 0, nullptr, out);
}

pgmg_status pgmg_dev_soln_diff(pgmg_handle* h, int level, const double* ext_x, double* out) {
    TRY(check_level(h, level));
    if (!out || !ext_x) return PGMG_ERR_ARG;
    const LevelGeom& g = h->L[level].g;
    CK(cudaMemcpyAsync(h->stage, ext_x, sizeof(double) * g.npts, cudaMemcpyDefault, h->stream));
    return helper_reduce(h, level, 1, h->stage, out);
}

pgmg_status pgmg_dev_l0_error(pgmg_handle* h, int level, double* out) {
    TRY(check_level(h, level));
    if (!out) return PGMG_ERR_ARG;
    return helper_reduce(h, level, 2, nullptr, out);
}

pgmg_status pgmg_dev_copy_r_to_x(pgmg_handle* h, int level) {
    TRY(check_level(h, level));
    h->x0_zero = false;
    Level& L = h->L[level];
    k_r_to_x<double><<<nblk(L.g.npts), kBlock, 0, h->stream>>>(L.g, L.r64, L.x64);
    CKL();
    return wrap_level<double>(h, level);
}

pgmg_status pgmg_dev_clear_x(pgmg_handle* h, int level) {
    TRY(check_level(h, level));
    if (level == 0) h->x0_zero = true;
    LAUNCH(nblk(h->L[level].g.npts), kBlock, k_clear_x<double>, h->L[level].g, h->L[level].x64);
    return wrap_level<double>(h, level);
}

pgmg_status pgmg_dev_setup_test(pgmg_handle* h, int level, int ca, int xfield) {
    TRY(check_level(h, level));
    h->x0_zero = false;
    Level& L = h->L[level];
    k_setup_test<double><<<nblk(L.g.npts), kBlock, 0, h->stream>>>(L.g, L.x64, L.r64, ca, xfield);
    CKL();
    return wrap_level<double>(h, level);
}

pgmg_status pgmg_dev_gs(pgmg_handle* h, int level, int mode, int smoother) {
    TRY(check_level(h, level));
    h->x0_zero = false;
    if (smoother < 0) smoother = h->dims.smoother;
    return gs_level<double>(h, level, mode, smoother, 1);
}

pgmg_status pgmg_dev_restrict(pgmg_handle* h, int level) {
    TRY(check_level(h, level));
    if (level < 1) return fail(h, PGMG_ERR_ARG, "restriction needs level >= 1");
    return restrict_level<double>(h, level);
}

pgmg_status pgmg_dev_interp(pgmg_handle* h, int level) {
    TRY(check_level(h, level));
    h->x0_zero = false;
    if (level < 1) return fail(h, PGMG_ERR_ARG, "interpolation needs level >= 1");
    return interp_level<double>(h, level);
}

pgmg_status pgmg_dev_coarse_solve(pgmg_handle* h) {
    if (!h) return PGMG_ERR_ARG;
    if (!h->built) return fail(h, PGMG_ERR_SETUP, "operators not built");
    if (h->nl == 1) h->x0_zero = false;
    return coarse_solve_t<double>(h, h->dims.smoother);
}

pgmg_status pgmg_dev_vcycle(pgmg_handle* h, int mode, int smoother) {
    if (!h) return PGMG_ERR_ARG;
    if (!h->built) return fail(h, PGMG_ERR_SETUP, "operators not built");
    if (smoother < 0) smoother = h->dims.smoother;
    h->x0_zero = false;
    if (h->dims.precision == PGMG_MIXED) return ir_step(h, mode, smoother, nullptr, nullptr);
    return run_vcycle<double>(h, mode, smoother);
}

}  // extern "C"

namespace {

// Autotuner state: the options chosen for a problem shape, remembered for
// the process.
struct TuneKey {
    int m, n, o, prd, precision, smoother, device;
    bool operator==(const TuneKey& b) const {
        return m == b.m && n == b.n && o == b.o && prd == b.prd && precision == b.precision &&
               smoother == b.smoother && device == b.device;
    }
};
struct TuneVal {
    int gs_block, coarse_first, cluster_size, pdl;
    long long grid_max;
    int gs_vec, gs_alt;
    long long gs_prefetch;
    int fused_restrict;
    long long gs_tma;
    long long gs_l2pf;
    long long gs_block_lv;
    double ms;
};
std::mutex g_tune_mu;
std::vector<std::pair<TuneKey, TuneVal>> g_tune;

void apply_tuning(pgmg_handle* h, const TuneVal& v) {
    h->gs_block = v.gs_block;
    h->coarse_first = v.coarse_first;
    h->cluster_size = v.cluster_size;
    h->pdl = v.pdl != 0;
    h->grid_max = v.grid_max;
    h->gs_vec = v.gs_vec;
    h->gs_alt = v.gs_alt != 0;
    h->gs_prefetch = v.gs_prefetch;
    h->fused_restrict = v.fused_restrict != 0;
    h->gs_tma = v.gs_tma;
    h->gs_l2pf = v.gs_l2pf;
    h->gs_block_lv = v.gs_block_lv;
    drop_graphs(h);
}

// Mean time of `reps` V-cycles (after one untimed cycle, which also captures
// the graph) under the handle's current options.
pgmg_status time_vcycles(pgmg_handle* h, int reps, cudaEvent_t e0, cudaEvent_t e1, double* ms) {
    drop_graphs(h);
    TRY(upload_plans(h));
    TRY(pgmg_dev_vcycle(h, 0, -1));
    CK(cudaEventRecord(e0, h->stream));
    for (int i = 0; i < reps; i++) TRY(pgmg_dev_vcycle(h, 0, -1));
    CK(cudaEventRecord(e1, h->stream));
    CK(cudaEventSynchronize(e1));
    TRY(check_grid(h));
    float t = 0;
    CK(cudaEventElapsedTime(&t, e0, e1));
    *ms = t / reps;
    return PGMG_OK;
}

}  // namespace

extern "C" {

pgmg_status pgmg_dev_grid_check(pgmg_handle* h, int level, int run_out) {
    TRY(check_level(h, level));
    if (h->grid_blocks[0] == 0) return fail(h, PGMG_ERR_UNSUPPORTED, "persistent sweep kernel not launchable");
    if (h->L[level].g.prd) return fail(h, PGMG_ERR_UNSUPPORTED, "periodic level");
    long long keep = h->grid_max;
    h->grid_max = 1;  // makes check_grid read the error word
    h->x0_zero = false;
    pgmg_status st = grid_sweeps<double>(h, level, 0, 1, run_out ? 1u : 0u);
    if (st == PGMG_OK) st = check_grid(h);
    h->grid_max = keep;
    return st;
}

pgmg_status pgmg_dev_profile_vcycle(pgmg_handle* h, int fp32, double* ms, int nms, int* first_coarse) {
    if (!h || !ms || nms < 4 * kMaxLevels + 1) return PGMG_ERR_ARG;
    if (!h->built) return fail(h, PGMG_ERR_SETUP, "operators not built");
    if (fp32 && h->dims.precision != PGMG_MIXED) return fail(h, PGMG_ERR_ARG, "fp32 profile needs a mixed handle");
    for (int q = 0; q < nms; q++) ms[q] = 0;
    TRY(upload_plans(h));
    std::vector<cudaEvent_t> ev;
    std::vector<int> tag;
    int lc = 0;
    h->x0_zero = false;
    pgmg_status st = fp32 ? vcycle_profiled<float>(h, h->dims.smoother, ev, tag, &lc)
                          : vcycle_profiled<double>(h, h->dims.smoother, ev, tag, &lc);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (st == PGMG_OK && e == cudaSuccess) {
        for (size_t q = 1; q < ev.size(); q++) {
            float t = 0;
            if (cudaEventElapsedTime(&t, ev[q - 1], ev[q]) == cudaSuccess) ms[tag[q]] += t;
        }
    }
    for (cudaEvent_t x : ev) cudaEventDestroy(x);
    if (first_coarse) *first_coarse = lc;
    TRY(st);
    CK(e);
    return check_grid(h);
}

pgmg_status pgmg_dev_tma_check(pgmg_handle* h, int level, int run_out) {
    TRY(check_level(h, level));
    const LevelGeom& g = h->L[level].g;
    if (g.prd) return fail(h, PGMG_ERR_UNSUPPORTED, "periodic level");
    long long keep = h->gs_tma;
    h->gs_tma = 1LL << 40;  // makes check_grid read the error word
    h->x0_zero = false;
    View<double> v = view<double>(h->L[level]);
    pgmg_status st = PGMG_OK;
    // One colour pass (with run_out, every CTA's wait runs out twice: about
    // a second for the pass).
    st = gs_tma_pass<double>(h, g, v, colour_seq(0), 0, (long)g.M2 * g.N2 * g.O2, run_out ? 16u : 0u);
    if (st == PGMG_OK) st = check_grid(h);
    h->gs_tma = keep;
    return st;
}

pgmg_status pgmg_dev_autotune(pgmg_handle* h, int reps, double* best_ms) {
    if (!h) return PGMG_ERR_ARG;
    TraceRange tr("pgmg autotune");
    if (!h->built) return fail(h, PGMG_ERR_SETUP, "operators not built");
    if (reps < 1) reps = 3;
    TuneKey key{h->dims.m, h->dims.n, h->dims.o, h->prd, h->dims.precision, h->dims.smoother, h->device};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        for (auto& kv : g_tune)
            if (kv.first == key) {
                apply_tuning(h, kv.second);
                TRY(upload_plans(h));
                if (best_ms) *best_ms = kv.second.ms;
                return PGMG_OK;
            }
    }
    // Save the level-0 solution (and whether it is known to be zero); the
    // timed V-cycles change it.
    Level& L0 = h->L[0];
    const LevelGeom& g0 = L0.g;
    bool zero = h->x0_zero;
    k_x_to_nat<double><<<nblk(g0.npts), kBlock, 0, h->stream>>>(g0, L0.x64, h->stage);
    CKL();
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    TuneVal best{h->gs_block,         h->coarse_first,   h->cluster_size, h->pdl ? 1 : 0,
                 h->grid_max,         h->gs_vec,         h->gs_alt ? 1 : 0, h->gs_prefetch,
                 h->fused_restrict ? 1 : 0, h->gs_tma, h->gs_l2pf, h->gs_block_lv, 0};
    pgmg_status st = time_vcycles(h, reps, e0, e1, &best.ms);
    // A candidate that times faster than the best so far is timed once more,
    // and so is the best, each keeping its faster time: the options differ
    // by a percent or two where they differ at all, about the run-to-run
    // spread of one timing.
    auto trial = [&](TuneVal c) -> pgmg_status {
        apply_tuning(h, c);
        double t = 0;
        pgmg_status s2 = time_vcycles(h, reps, e0, e1, &t);
        if (s2 == PGMG_ERR_TIMEOUT) return PGMG_OK;  // a candidate that fails is not kept
        if (s2 != PGMG_OK) return s2;
        if (t < best.ms) {
            double tb = 0, tc = 0;
            apply_tuning(h, best);
            if ((s2 = time_vcycles(h, reps, e0, e1, &tb)) != PGMG_OK) return s2;
            apply_tuning(h, c);
            s2 = time_vcycles(h, reps, e0, e1, &tc);
            if (s2 == PGMG_ERR_TIMEOUT) return PGMG_OK;
            if (s2 != PGMG_OK) return s2;
            if (tb < best.ms) best.ms = tb;
            if (tc < t) t = tc;
        }
        c.ms = t;
        if (t < best.ms) best = c;
        return PGMG_OK;
    };
    bool mc8 = h->dims.smoother == PGMG_SMOOTH_MC8;
    // Coordinate descent: one option at a time, each from the best so far.
    if (st == PGMG_OK && mc8) {
        TuneVal c = best;
        c.gs_alt = !best.gs_alt;
        st = trial(c);
    }
    if (st == PGMG_OK && mc8 && !h->prd) {
        long long p0 = best.gs_prefetch;
        for (long long pm : {0LL, 1LL << 18, 1LL << 22, 1LL << 26}) {
            if (st != PGMG_OK || pm == p0) continue;
            TuneVal c = best;
            c.gs_prefetch = pm;
            st = trial(c);
        }
    }
    if (st == PGMG_OK && mc8 && !h->prd) {
        // 2 points per thread differs from 16-byte vectors only in FP32.
        const int vmax = h->dims.precision == PGMG_MIXED ? 2 : 1;
        const int v0 = best.gs_vec;
        for (int vv = 0; vv <= vmax && st == PGMG_OK; vv++) {
            if (vv == v0) continue;
            TuneVal c = best;
            c.gs_vec = vv;
            st = trial(c);
        }
    }
    if (st == PGMG_OK && mc8 && !h->prd) {
        long long q0 = best.gs_l2pf;
        for (long long lp : {0LL, 1LL << 19, 1LL << 22}) {
            if (st != PGMG_OK || lp == q0) continue;
            TuneVal c = best;
            c.gs_l2pf = lp;
            st = trial(c);
        }
    }
    if (st == PGMG_OK && mc8 && !h->prd) {
        long long t0 = best.gs_tma;
        for (long long tm : {0LL, 1LL << 19, 1LL << 22, 1LL << 26}) {
            if (st != PGMG_OK || tm == t0) continue;
            TuneVal c = best;
            c.gs_tma = tm;
            st = trial(c);
        }
    }
    if (st == PGMG_OK && mc8 && !h->prd)
        for (int b : {128, 256, 512}) {
            if (b == best.gs_block) continue;
            TuneVal c = best;
            c.gs_block = b;
            if ((st = trial(c)) != PGMG_OK) break;
        }
    if (st == PGMG_OK && mc8 && h->cluster_size > 0 && h->dims.coarse != PGMG_COARSE_LU_EXACT) {
        int f0 = best.coarse_first;
        for (int l = 0; l <= h->nl && st == PGMG_OK; l++) {
            if (l == f0 || (l < h->nl && h->L[l].g.npts > 6 * kClusterMax)) continue;
            TuneVal c = best;
            c.coarse_first = l;
            st = trial(c);
        }
        int s0 = best.cluster_size;
        for (int cs : {1, 2, 4, 8, 16}) {
            if (st != PGMG_OK || cs == s0 || probe_cluster<double>(cs) <= 0 || probe_cluster<float>(cs) <= 0) continue;
            TuneVal c = best;
            c.cluster_size = cs;
            st = trial(c);
        }
        // A smaller cluster may prefer a lower first level: try its neighbours.
        if (st == PGMG_OK && best.cluster_size != s0) {
            int f1 = best.coarse_first;
            for (int l : {f1 - 1, f1 + 1}) {
                if (l < 0 || l > h->nl || (l < h->nl && h->L[l].g.npts > 6 * kClusterMax)) continue;
                TuneVal c = best;
                c.coarse_first = l;
                if ((st = trial(c)) != PGMG_OK) break;
            }
        }
    }
    // Block size per swept level above the cluster tail (a level's best can
    // differ from level 0's: at 257^3 FP64, 512 threads on 129^3 and 128 on
    // 33^3).
    if (st == PGMG_OK && mc8 && !h->prd) {
        const int top = best.coarse_first < h->nl ? best.coarse_first : h->nl;
        for (int l = 1; l < top && l <= 15 && st == PGMG_OK; l++)
            for (int code = 1; code <= 3 && st == PGMG_OK; code++) {
                const int sh = 2 * (l - 1);
                const int cur = (int)((best.gs_block_lv >> sh) & 3);
                const int size = code == 1 ? 128 : code == 2 ? 256 : 512;
                const int cur_size = cur == 0 ? best.gs_block : cur == 1 ? 128 : cur == 2 ? 256 : 512;
                if (size == cur_size) continue;
                TuneVal c = best;
                c.gs_block_lv = (best.gs_block_lv & ~(3LL << sh)) | ((long long)code << sh);
                st = trial(c);
            }
    }
    if (st == PGMG_OK && mc8 && !h->prd && h->grid_blocks[0] > 0 && h->grid_blocks[1] > 0) {
        long long g0 = best.grid_max;
        for (long long gm : {0LL, 300000LL, 3000000LL, 30000000LL}) {
            if (gm == g0) continue;
            TuneVal c = best;
            c.grid_max = gm;
            if ((st = trial(c)) != PGMG_OK) break;
        }
    }
    if (st == PGMG_OK && !h->prd) {
        TuneVal c = best;
        c.fused_restrict = !best.fused_restrict;
        st = trial(c);
    }
    if (st == PGMG_OK) {
        TuneVal c = best;
        c.pdl = !best.pdl;
        st = trial(c);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    apply_tuning(h, best);
    TRY(upload_plans(h));
    // Restore the solution.
    k_nat_to_x<double><<<nblk(g0.npts), kBlock, 0, h->stream>>>(g0, h->stage, L0.x64);
    CKL();
    TRY(wrap_level<double>(h, 0));
    CK(cudaStreamSynchronize(h->stream));
    h->x0_zero = zero;
    if (st != PGMG_OK) return st;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune.push_back({key, best});
    }
    if (best_ms) *best_ms = best.ms;
    return PGMG_OK;
}

pgmg_status pgmg_dev_fmg_cycle(pgmg_handle* h, int smoother) {
    if (!h) return PGMG_ERR_ARG;
    if (!h->built) return fail(h, PGMG_ERR_SETUP, "operators not built");
    if (smoother < 0) smoother = h->dims.smoother;
    TraceRange tr("pgmg fmg_cycle");
    h->x0_zero = false;
    // multigrid::fmg_cycle (multigrid.cc:109-134), mode 0.
    int ml = h->nl;
    for (int i = 0; i < ml - 1; i++) {
        TRY(restrict_level<double>(h, i + 1));
        TRY(gs_level<double>(h, i + 1, 0, smoother, h->v_down));
    }
    for (int j = ml - 1; j > 0; j--) {
        for (int i = j; i < ml - 1; i++) {
            TRY(restrict_level<double>(h, i + 1));
            TRY(gs_level<double>(h, i + 1, 0, smoother, h->v_down));
        }
        TRY(gs_level<double>(h, ml - 1, 0, smoother, h->v_bottom));
        for (int i = ml - 1; i >= j; i--) {
            TRY(interp_level<double>(h, i));
            TRY(gs_level<double>(h, i - 1, 0, smoother, h->v_up));
        }
    }
    return PGMG_OK;
}

pgmg_status pgmg_dev_norms(pgmg_handle* h, int level, double* res2, double* rhs2) {
    TRY(check_level(h, level));
    TraceRange tr("pgmg norms");
    return norms64(h, level, res2, rhs2);
}

pgmg_status pgmg_dev_solve_v_cycles(pgmg_handle* h, double p_scale, int* result, double* res2, int* cycles) {
    if (!h) return PGMG_ERR_ARG;
    if (!h->built) return fail(h, PGMG_ERR_SETUP, "operators not built");
    TraceRange tr("pgmg solve_v_cycles");
    if (!h->tol_set) {
        if (!(p_scale > 0)) return fail(h, PGMG_ERR_SETUP, "solve_v_cycles needs guide.set_tol (p_scale > 0)");
        double eps = 2.220446049250313e-16;
        h->tol = p_scale * p_scale * eps * eps * 10000;
        h->tol_set = 1;
    }
    double tol = h->tol * h->dims.m;
    tol *= h->dims.n;
    tol *= h->dims.o;
    int nc = 0;
    int pred = h->iter / h->period;
    for (int i = 0; i < pred; i++, nc++) TRY(pgmg_dev_vcycle(h, 0, -1));
    int extra = 0, n = 0;
    double res = 0;
    int st = 0;
    // The reference's loop (multigrid.hh:202-210): a NaN residual fails the
    // "res > tol" test and leaves the loop, so its NaN branch is never taken
    // and such a solve reports 0; this loop keeps that behaviour.
    for (;;) {
        TRY(norms64(h, 0, &res, nullptr));
        if (!(res > tol && n < 100)) break;
        if (std::isnan(res)) { st = 2; break; }
        extra++;
        for (int i = 0; i < extra; i++, n++, nc++) TRY(pgmg_dev_vcycle(h, 0, -1));
    }
    if (st == 0 && n > 100) st = 1;
    if (st == 0) {
        for (int i = 0; i < 2; i++, nc++) TRY(pgmg_dev_vcycle(h, 0, -1));
        guide_update(h, extra * (extra + 1) / 2);
    }
    if (result) *result = st;
    if (res2) *res2 = res;
    if (cycles) *cycles = nc;
    return check_grid(h);
}

// Residual-check schedule of the relative-residual solve.  check_every >= 1:
// every that many cycles.  check_every == 0: adaptive -- the per-cycle
// reduction factor is estimated from the last two checks (or remembered from
// the handle's previous solve) and the solve runs the cycles predicted to
// reach tol before checking again, stopping one short when that one might
// already be enough.

struct CheckPlan {
    int every;
    double rho0 = 0;  // reduction factor remembered from an earlier solve
    int last_n = -1, prev_n = -1, first_n = -1;
    double last_r = 0, prev_r = 0, first_r = 0;
    double rho() const {
        if (prev_n >= 0 && last_r > 0 && prev_r > 0) return pow(last_r / prev_r, 1.0 / (last_n - prev_n));
        return rho0;
    }
    int next(int nc, double tol) const {
        if (every >= 1) return nc + every;
        double q = rho();
        if (!(q > 0) || q >= 0.9 || !(last_r > 0)) return nc + 1;
        double need = log(tol / last_r) / log(q);
        int n = (int)ceil(need);
        if (n < 1) n = 1;
        // The reduction factor is an estimate: when the cycle before the
        // predicted one might already reach tol (its predicted residual is
        // within kSlack of tol), check after it -- a check costs a fraction
        // of a cycle, a needless cycle costs a whole one.
        if (n > 1 && last_r * pow(q, n - 1) < kSlack * tol) n--;
        return nc + n;
    }
    void record(int nc, double r) {
        if (first_n < 0) { first_n = nc; first_r = r; }
        prev_n = last_n; prev_r = last_r; last_n = nc; last_r = r;
    }
};


// The solve of pgmg_dev_solve_relres.  x_out (pgmg_dev_solve_io; may be
// NULL): the caller's buffer for the level-0 solution in natural order.  At
// a check that may end the solve the solution is converted and copied there
// on the handle's output stream while the check itself runs on the handle's
// stream; if the check does not end the solve, a later copy on the same
// stream follows the stale one.
static pgmg_status solve_core(pgmg_handle* h, double tol, int max_cycles, int check_every, int* cycles,
                              double* relres, double* x_out) {
    if (!h) return PGMG_ERR_ARG;
    if (!h->built) return fail(h, PGMG_ERR_SETUP, "operators not built");
    TraceRange tr("pgmg solve");
    if (check_every < 0) check_every = 1;
    int smoother = h->dims.smoother;
    double res2 = 0, rhs2 = 0, rr = INFINITY;
    int nc = 0, next_check = 0;
    CheckPlan plan;
    plan.every = check_every;
    Level& L0 = h->L[0];
    const LevelGeom& g = L0.g;
    dim3 grid((unsigned)(8 * nblk((long)g.M2 * g.N2 * g.O2)));  // colours interleaved
    long nb = nblk((long)g.M2 * g.N2 * g.O2) * 8;
    bool mixed = h->dims.precision == PGMG_MIXED;
    bool spec64 = false, out_now = false;
    plan.rho0 = h->last_rho;
    for (;;) {
        // Mixed precision computes the FP64 residual at every refinement step
        // (it is the next correction's source), so it checks every step too.
        bool check = mixed || nc >= next_check || nc >= max_cycles;
        bool zero = nc == 0 && h->x0_zero;  // residual = source: no stencil pass needed
        TraceRange check_range("pgmg check", check);  // ends once the norms are read
        out_now = false;
        if (x_out && check && !zero) {
            // An FP64 check is scheduled where the solve is predicted to
            // converge; a mixed one ends the solve unless its predicted
            // residual is above kSlack * tol.
            bool more = false;
            if (mixed) {
                double q = plan.rho();
                more = q > 0 && q < 0.9 && plan.last_r > 0 && plan.last_r * pow(q, nc - plan.last_n) > kSlack * tol;
            }
            if (!more) {
                CK(cudaEventRecord(h->ev_out, h->stream));
                CK(cudaStreamWaitEvent(h->ostream, h->ev_out, 0));
                k_x_to_nat<double><<<nblk(g.npts), kBlock, 0, h->ostream>>>(g, L0.x64, h->stage);
                CKL();
                CK(cudaMemcpyAsync(x_out, h->stage, sizeof(double) * g.npts, cudaMemcpyDefault, h->ostream));
                out_now = true;
            }
        }
        if (check) TRY(check_begin(h));
        if (zero) {
            if (mixed || check) {
                LAUNCH(grid, kBlock, k_source<double, float>, g, L0.r64, mixed ? L0.r32 : nullptr, h->partials);
            }
        } else if (mixed) {
            // FP64 residual of the current x, stored FP32 as the correction's
            // source (and reduced to the norms when checking).
            LAUNCH(grid, kBlock, k_residual<double, float, true>, g, L0.x64, L0.r64, L0.A64, L0.r32,
                                                                              check ? h->partials : nullptr);
        } else if (check) {
            LAUNCH(grid, kBlock, k_residual<double, double, true>, g, L0.x64, L0.r64, L0.A64, nullptr,
                                                                               h->partials);
        }
        // Mixed precision: when this check is expected to find the solve not
        // yet converged, the next refinement step's first FP32 V-cycle (which
        // changes only the correction e, never x64) is enqueued before the
        // host waits for the norms, so the GPU does not idle during the round
        // trip.  If the check converges after all, that work is simply not
        // used; the result is the same either way.
        bool spec = false;
        if (check && mixed) {
            TRY(reduce_launch(h, nb));
            if (nc < max_cycles) {
                if (zero) {
                    spec = tol < 1.0;  // x = 0: the relative residual is 1 (unless the source is 0)
                } else {
                    double q = plan.rho();
                    spec = q > 0 && q < 0.9 && plan.last_r > 0 &&
                           plan.last_r * pow(q, nc - plan.last_n) > kSlack * tol;
                }
            }
            if (spec) {
                CK(cudaMemsetAsync(L0.x32, 0, g.xsize() * sizeof(float), h->stream));
                TRY(wrap_level<float>(h, 0));
                TRY(run_vcycle<float>(h, 0, smoother));
            }
            TRY(read_norms(h));
        } else if (check) {
            // FP64 from x = 0: the check is the source norm, which ends the
            // solve only for a zero or non-finite source (or tol >= 1), so
            // the first V-cycle is enqueued before the host waits for it;
            // when the solve does end there, x is cleared again.
            TRY(reduce_launch(h, nb));
            if (zero && nc < max_cycles && tol < 1.0) {
                TRY(run_vcycle<double>(h, 0, smoother));
                spec64 = true;
            }
            TRY(read_norms(h));
        }
        if (check) {
            res2 = h->norm_host[0];
            rhs2 = h->norm_host[1];
            rr = rhs2 > 0 ? sqrt(res2 / rhs2) : sqrt(res2);
            if (std::isnan(rr) || rr < tol || nc >= max_cycles) {
                if (spec64) TRY(pgmg_dev_clear_x(h, 0));
                if (spec64) out_now = false;
                break;
            }
            plan.record(nc, rr);
            next_check = plan.next(nc, tol);
            if (next_check > max_cycles) next_check = max_cycles;
        }
        check_range.end();
        h->x0_zero = false;
        if (mixed) {
            TraceRange step_range("pgmg refinement step");
            // One refinement step: A32 e = r32 solved by `inner` FP32
            // V-cycles from e = 0, then x64 += e.  The count is the number of
            // cycles the check schedule expects to run before its next check;
            // with the adaptive schedule it is limited by ir_inner_cycles to
            // what one FP32 solve can usefully reduce.
            int inner = next_check - nc;
            if (plan.every == 0) inner = ir_inner_cycles(inner, plan.rho(), h->inner_digits);
            if (inner > max_cycles - nc) inner = max_cycles - nc;
            if (inner < 1) inner = 1;
            if (!spec) {
                CK(cudaMemsetAsync(L0.x32, 0, g.xsize() * sizeof(float), h->stream));  // e = 0 (halo too)
                TRY(wrap_level<float>(h, 0));
            }
            for (int i = spec ? 1 : 0; i < inner; i++) TRY(run_vcycle<float>(h, 0, smoother));
            TRY(add_correction(h));
            TRY(wrap_level<double>(h, 0));
            nc += inner;
            continue;
        } else if (spec64) {
            spec64 = false;  // this cycle was enqueued before the check was read
        } else {
            TRY(run_vcycle<double>(h, 0, smoother));
        }
        nc++;
    }
    // Remember the mean reduction per cycle over the whole solve: the next
    // solve starts from its own first residual, and multigrid usually
    // reduces faster in the first cycles than later, so the last interval's
    // factor alone would overestimate the cycles a fresh solve needs.
    if (nc > plan.first_n && plan.first_n >= 0 && plan.first_r > 0 && rr > 0) {
        double q = pow(rr / plan.first_r, 1.0 / (nc - plan.first_n));
        if (q > 0 && q < 0.9) h->last_rho = q;
    }
    if (x_out) {
        // The copy enqueued at the final check holds the final x; otherwise
        // (the solve ended at x = 0, or without a copy) copy it now.
        CK(cudaStreamSynchronize(h->ostream));
        if (!out_now) {
            k_x_to_nat<double><<<nblk(g.npts), kBlock, 0, h->stream>>>(g, L0.x64, h->stage);
            CKL();
            CK(cudaMemcpyAsync(x_out, h->stage, sizeof(double) * g.npts, cudaMemcpyDefault, h->stream));
            CK(cudaStreamSynchronize(h->stream));
        }
    }
    if (cycles) *cycles = nc;
    if (relres) *relres = rr;
    return check_grid(h);
}

pgmg_status pgmg_dev_solve_relres(pgmg_handle* h, double tol, int max_cycles, int check_every, int* cycles,
                                  double* relres) {
    return solve_core(h, tol, max_cycles, check_every, cycles, relres, nullptr);
}

pgmg_status pgmg_dev_solve_io(pgmg_handle* h, const double* r, double* x, double tol, int max_cycles,
                              int check_every, int* cycles, double* relres) {
    if (!h || !r || !x) return PGMG_ERR_ARG;
    if (!h->built) return fail(h, PGMG_ERR_SETUP, "operators not built");
    TraceRange tr("pgmg solve_io");
    if (!h->ostream) {
        if (cudaStreamCreateWithFlags(&h->ostream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->ev_out, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return fail(h, PGMG_ERR_CUDA, "output stream");
        }
    }
    Level& L0 = h->L[0];
    const LevelGeom& g = L0.g;
    CK(cudaMemcpyAsync(h->stage, r, sizeof(double) * g.npts, cudaMemcpyDefault, h->stream));
    k_nat_to_cm<double><<<nblk(g.npts), kBlock, 0, h->stream>>>(g, h->stage, L0.r64);
    CKL();
    TRY(pgmg_dev_clear_x(h, 0));
    const pgmg_status st = solve_core(h, tol, max_cycles, check_every, cycles, relres, x);
    // On an error return too, no copy into the caller's buffer may still be
    // in flight.
    if (st != PGMG_OK && cudaStreamSynchronize(h->ostream) != cudaSuccess) cudaGetLastError();
    return st;
}

}  // extern "C"
