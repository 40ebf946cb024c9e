// Internal: the handle behind pgmg_handle* and its per-level buffers, shared
// by the single-problem entry points (capi.cu) and the batched solver
// (batch.cu).
#pragma once
#include <utility>

#include "../../include/pgmg_dev.h"
#include "kernels_coarse.cuh"
#include "kernels_core.cuh"
#include "kernels_grid.cuh"
#include "kernels_setup.cuh"
#include "kernels_tma.cuh"
#include "layout.cuh"
#include "trace.cuh"

namespace pgmg {
constexpr int kMaxLevels = 16;      // mg_max_levels, common.hh:15
constexpr int kGsExact = 24;        // pgmg_gs_exact, common.hh:62
constexpr int kMaxExact = 2048;     // pgmg_max_exact, common.hh:65
constexpr long kLexBlockMax = 40000;  // levels up to this size sweep lexicographically in one block
constexpr long kMc8BlockMax = 10000;  // levels up to this size sweep 8 colours in one block
constexpr long kClusterMax = 50000;   // levels up to this size run in the one-cluster coarse cycle
constexpr int kClusterThreads = 512;
constexpr int kCoarseXsMax = 200 * 1024;  // dynamic shared memory for a coarse level's x copy
// Residual-check schedule (single solves and batches): check one cycle
// before the predicted count when that cycle's predicted residual is within
// kSlack of tol.  Mixed precision: the reduction (in decimal digits) asked of
// the FP32 V-cycles of one refinement step by default, and the most cycles
// one step runs.
constexpr double kSlack = 3.0;
constexpr int kInnerDigits = 5;
constexpr int kInnerMax = 16;

// FP32 V-cycles of one mixed-precision refinement step, given the `want`
// cycles the schedule predicts to reach the tolerance and the estimated
// reduction q per cycle.  A step asks the FP32 iteration for at most a
// 10^-digits reduction (beyond that FP32 rounding, not the cycle count,
// limits what the correction gains); a solve that gains at least a digit per
// cycle (q < 0.1, a well-conditioned operator) asks one digit more, so that
// its few cycles split into fewer refinement steps, each of which costs an
// FP64 residual pass and a host round trip.  Measured at 257^3: sigma = 1
// (q ~ 0.04) 7 cycles in two steps instead of three, 3 % faster; sigma = 2.3
// (q ~ 0.4) keeps 5 digits, where asking 6 took 26 cycles instead of 24.
__host__ __device__ inline int ir_inner_cycles(int want, double q, int digits) {
    if (!(q > 0) || q >= 0.9) return 1;
    const int d = q < 0.1 ? digits + 1 : digits;
    int cap = (int)floor(-d * log(10.0) / log(q));
    cap = cap < 1 ? 1 : cap > kInnerMax ? kInnerMax : cap;
    return want < cap ? want : cap;
}

struct Level {
    LevelGeom g;
    double *A64 = nullptr, *x64 = nullptr, *r64 = nullptr, *res64 = nullptr;
    float *A32 = nullptr, *x32 = nullptr, *r32 = nullptr, *res32 = nullptr;
    int8_t* S = nullptr;
};

template <class T> struct View { T *A, *x, *r, *res; };
inline View<double> view64(Level& L) { return {L.A64, L.x64, L.r64, L.res64}; }
inline View<float> view32(Level& L) { return {L.A32, L.x32, L.r32, L.res32}; }

__host__ __device__ inline long nblk(long n, int b = kBlock) { return (n + b - 1) / b; }

// Simple bump allocator over one device allocation (256-byte aligned).
struct Arena {
    char* base = nullptr;
    size_t size = 0, used = 0;
    template <class T> T* take(size_t count) {
        size_t bytes = (count * sizeof(T) + 255) / 256 * 256;
        T* p = base ? reinterpret_cast<T*>(base + used) : nullptr;
        used += bytes;
        return p;
    }
};

// Launches k(args...) on `stream`; with `pdl` set, as a programmatic
// dependent launch (k must start with pdl_enter(): it may be scheduled while
// the previous kernel of the stream drains, and waits there for it).
template <typename... KArgs, typename... Args>
cudaError_t launch_k(cudaStream_t stream, bool pdl, dim3 grid, dim3 block, void (*k)(KArgs...), Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}

// launch_k with dynamic shared memory.
template <class... KArgs, class... Args>
cudaError_t launch_k_smem(cudaStream_t stream, bool pdl, dim3 grid, dim3 block, size_t smem, void (*k)(KArgs...),
                          Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}

}  // namespace pgmg

struct pgmg_handle {
    using Level = pgmg::Level;
    using Arena = pgmg::Arena;
    pgmg_dims dims{};
    int device = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    int nl = 0;
    Level L[pgmg::kMaxLevels];
    Arena arena;
    // coarsest level
    long nex = 0;
    double *M = nullptr, *Minv = nullptr, *lubuf = nullptr;
    int *piv = nullptr, *info = nullptr;
    int lu_ok = 0;
    bool uploaded = false, built = false;
    // staging and reductions
    double* stage = nullptr;
    size_t stage_elems = 0;
    double* partials = nullptr;
    double* norm_dev = nullptr;
    double norm_host[2] = {0, 0};
    // Residual checks: the reduction writes the two norms straight into this
    // pinned host pair (null if it could not be had: then they are copied
    // from norm_dev); ev_pre is recorded before the check's residual kernel,
    // ev_post after the reduction.
    double* norm_pin = nullptr;
    cudaEvent_t ev_pre = nullptr, ev_post = nullptr;
    // pgmg_dev_solve_io: the solution's copy to the caller's buffer runs on
    // ostream (created at the first call), after ev_out on the handle's stream.
    cudaStream_t ostream = nullptr;
    cudaEvent_t ev_out = nullptr;
    bool own_arena = true;         // false: memory given by the caller
    // mg_guide state (multigrid.hh:34-118)
    int period = 16, iter = 16, use_avg = 0, tol_set = 0;
    double iter_avg = 16, iter_var = 1000000, alpha = 3.0 / 16, tol = 0;
    long long launches = 0;  // kernels this handle has launched
    bool x0_zero = true;     // level-0 x known to be zero (cleared, not written since)
    double last_rho = 0;     // per-cycle residual reduction seen by the last solve
    // Captured V-cycles, by [float][mode][smoother].
    cudaGraphExec_t vgraph[2][2][2] = {};
    long long vgraph_nodes[2][2][2] = {};
    bool use_graphs = true;
    int prd = 0;      // periodic axes of the problem (bit 0 x, 1 y, 2 z)
    bool pdl = true;
    int gs_block = 256;  // threads per block of the colour sweep
    int gs_vec = 0;  // colour sweep with vector loads (k_gs_colour_v): 1 = 16-byte, 2 = 2 points per thread
    bool gs_alt = true;   // colour passes alternate their traversal direction
    // 8-colour levels of at most gs_prefetch points load their stencil before
    // the launch dependency (k_gs_colour_pf); 0 = none.  On the largest
    // levels the extra registers cost more occupancy than the overlap wins.
    long long gs_prefetch = 1LL << 22;
    // Coarse-cycle sweeps keep the level's x in each CTA's shared memory
    // (levels whose halo'd x fits in kCoarseXsMax bytes).
    bool coarse_shared = true;
    // Non-periodic restrictions compute their residuals inside the kernel
    // (k_resrestrict) instead of a residual pass plus k_restrict_fast; off by
    // default (slower, measured), tried by the autotuner.
    bool fused_restrict = false;
    // 8-colour levels of at most gs_tma points (one slab, non-periodic)
    // stage each pass's stencils and sources with bulk copies
    // (k_gs_colour_tma); 0 = off.
    long long gs_tma = 0;
    // The coarse LU factorises in a shared-memory band window (k_lu_window)
    // where it fits, instead of the one-block kernel on device memory.
    bool lu_window = true;
    // The explicit coarse inverse one warp per column over the factors' band
    // (k_lu_inverse_band) where the band allows, instead of k_lu_inverse.
    bool lu_inv_band = true;
    // Galerkin operators of large non-periodic levels by k_rat_tile (one
    // thread per coarse point and slot) instead of k_rat_fill (off: measured
    // slower).
    bool rat_tile = false;
    // k_gs_colour_pf levels of at most gs_l2pf points prefetch the next
    // pass's stencils into L2 (0 = off).
    long long gs_l2pf = 0;
    // Per-level block sizes of the colour sweep: 2 bits per level 1..15
    // (bits 2l-2, 2l-1): 0 = gs_block, 1/2/3 = 128/256/512 threads.
    long long gs_block_lv = 0;
    int inner_digits = pgmg::kInnerDigits;  // mixed precision: reduction asked of one refinement step (ir_inner_cycles)
    // Persistent whole-GPU sweeps (k_sweeps_grid) for levels above the
    // cluster levels with at most grid_max points (0 = off); co-resident
    // blocks of 512 threads per precision (0 = not launchable).
    long long grid_max = 0;
    int grid_blocks[2] = {0, 0};
    pgmg::GridBar* bar = nullptr;  // V-cycle and solve-loop kernels as programmatic dependent launches
    // One-cluster coarse cycle: CTAs per cluster (0 = unavailable) and the
    // first level it handles.
    int cluster_size = 0;
    int coarse_first = 0;
    long long slab_budget = 0;  // bytes of x per slab of the 8-colour sweep (0 = one slab)
    // Device copies of the coarse-cycle plans (CoarsePlan<double>, <float>).
    pgmg::CoarsePlan<double>* plan64 = nullptr;
    pgmg::CoarsePlan<float>* plan32 = nullptr;
    // Public sweep counts of the reference's multigrid (multigrid.hh:122-128).
    int v_down = 2, v_up = 2, v_bottom = 20;
    char err[512] = {0};
};

