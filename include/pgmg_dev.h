/* pgmg_dev.h -- C ABI of the B200 geometric multigrid library (libpgmg_b200.so).
 *
 * Plain pointers, sizes and status codes; no C++ or torch types.  The C++
 * drop-in headers (include/pgmg/multigrid.hh and friends) sit on top of this
 * ABI and keep the reference's class interface; a ctypes binding
 * (pgmg_b200/__init__.py) calls it from Python.
 *
 * Scope: one process, one GPU, the whole level hierarchy resident in device
 * memory.  Each entry point names the reference interface it replaces
 * (file:line in chr1shr/pgmg).
 *
 * Conventions
 *   - Grids are m x n x o nodes; arrays are natural order, i fastest.
 *   - Stencils: 27 slots per point, slot (di+1)+3*(dj+1)+9*(dk+1) for the
 *     neighbour at offset (di,dj,dk) in {-1,0,1}^3; entries outside the
 *     point's box are zero.  Boxes ("S", region.hh:252-256) are 6 ints per
 *     point [xd,xu,yd,yu,zd,zu] relative to the point and must lie inside
 *     [-1,2)^3 and inside the grid on non-periodic axes.
 *   - Host/device: every array argument may be host memory (pageable or
 *     pinned) or device memory of the handle's GPU; the library tells them
 *     apart through unified addressing.
 *   - Ownership: the handle owns all device memory it allocates; caller
 *     pointers are borrowed for the duration of the call only.  The
 *     reference aliases external_ptr stencils for the multigrid lifetime
 *     (region.hh:517); this library copies them at upload instead.
 *   - Streams: all work of a handle is issued on one CUDA stream (its own,
 *     or the one given to pgmg_dev_set_stream).  Calls returning host values
 *     synchronise that stream.  One handle is not thread-safe; different
 *     handles may be used from different threads.
 *   - Errors: every call returns a pgmg_status; nothing aborts.  The C++
 *     drop-in maps a non-zero status to p_fatal_error (common.cc:52-55)
 *     except where the reference itself returns codes.
 */
#ifndef PGMG_DEV_H
#define PGMG_DEV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  1..6 mirror the reference's error enum (common.hh:19-26,
 * PGMG_FILE_ERROR..PGMG_SETUP_ERROR, shifted by one so that 0 is success). */
typedef enum {
    PGMG_OK = 0,
    PGMG_ERR_FILE = 1,
    PGMG_ERR_MEMORY = 2,
    PGMG_ERR_INTERNAL = 3,
    PGMG_ERR_MULTIGRID = 4,
    PGMG_ERR_MATH = 5,
    PGMG_ERR_SETUP = 6,
    PGMG_ERR_ARG = 7,          /* bad argument or unsupported stencil box   */
    PGMG_ERR_CUDA = 8,         /* a CUDA runtime call failed                */
    PGMG_ERR_TIMEOUT = 9,      /* a bounded device wait ran out             */
    PGMG_ERR_ADMISSION = 10,   /* request does not fit the memory cap       */
    PGMG_ERR_UNSUPPORTED = 11, /* configuration not supported (e.g. the Q1
                                  generator on a periodic grid)            */
    PGMG_ERR_NO_DEVICE = 12    /* no CUDA device visible                    */
} pgmg_status;

/* Smoother of a sweep. */
enum {
    PGMG_SMOOTH_MC8 = 0, /* 8-colour Gauss-Seidel, colours (i&1)|(j&1)<<1|(k&1)<<2
                            swept in the order 0,6,5,3,7,1,2,4 (even i+j+k first) */
    PGMG_SMOOTH_LEX = 1  /* lexicographic order as region.cc:367-446, by wavefronts */
};

/* Coarsest-level solver. */
enum {
    PGMG_COARSE_LU = 0,  /* FP64 LU with the reference's conditioning check
                            (region_tr.cc:483-534); falls back to GS if it fails */
    PGMG_COARSE_GS = 1,  /* always pgmg_gs_exact=24 lexicographic sweeps, the
                            reference's fallback path (region_tr.cc:557) */
    PGMG_COARSE_LU_EXACT = 2 /* LU solved in DGETRS order (one thread block), bit
                            for bit the reference's solve; slower than the
                            explicit-inverse product PGMG_COARSE_LU uses */
};

/* Arithmetic of the V-cycle. */
enum {
    PGMG_FP64 = 0,       /* all-FP64, the drop-in */
    PGMG_MIXED = 1       /* FP64 iterative refinement around an FP32 V-cycle */
};

/* Fields of a level. */
enum {
    PGMG_FIELD_X = 0,    /* solution x (region.hh:50-53) */
    PGMG_FIELD_R = 1,    /* source r   (region.hh:55)    */
    PGMG_FIELD_RES = 2   /* residual r - A x (read only) */
};

typedef struct pgmg_handle pgmg_handle;

/* Grid and options.  Replaces geometry(m,n,o,x_prd,y_prd,z_prd)
 * (geometry.cc:12-26) on one process, plus the run-time choices. */
typedef struct {
    int m, n, o;              /* global grid size                          */
    int x_prd, y_prd, z_prd;  /* periodicity (non-zero: periodic; any size,
                                 coarse size (m+1)>>1, region.cc:14)      */
    int precision;            /* PGMG_FP64 or PGMG_MIXED                    */
    int coarse;               /* PGMG_COARSE_LU or PGMG_COARSE_GS           */
    int smoother;             /* default smoother of pgmg_dev_vcycle        */
    int device;               /* CUDA device ordinal, -1 = current          */
} pgmg_dims;

/* ---- lifetime -------------------------------------------------------- */

/* Plans the hierarchy (multigrid::setup_hierarchy, multigrid.cc:17-85: coarsen
 * by (m+2)>>1 while m*n*o > 1024) and allocates every level in one device
 * arena.  Replaces multigrid(p_class&,geometry&,comm_buffer&)
 * (multigrid.hh:283-295) minus the problem-class callbacks. */
pgmg_status pgmg_dev_create(const pgmg_dims *dims, pgmg_handle **out);
/* As pgmg_dev_create, but the handle lives inside caller-owned device memory
 * `mem` (256-byte aligned, at least pgmg_dev_plan_bytes bytes) and never
 * allocates or frees device memory itself -- for servers that manage one
 * pool and must not stall the device in cudaMalloc/cudaFree. */
pgmg_status pgmg_dev_create_in(const pgmg_dims *dims, void *mem, size_t bytes, pgmg_handle **out);
/* Frees everything (multigrid::~multigrid, multigrid.cc:7-14). */
pgmg_status pgmg_dev_destroy(pgmg_handle *h);
/* Issue all further work of the handle on this cudaStream_t (NULL = the
 * handle's own stream). */
pgmg_status pgmg_dev_set_stream(pgmg_handle *h, void *cuda_stream);
/* Waits for all work of the handle. */
pgmg_status pgmg_dev_sync(pgmg_handle *h);
/* Text of the last error on this handle (static storage, never NULL). */
const char *pgmg_dev_last_error(pgmg_handle *h);
/* Kernels the handle has launched so far (all of them this library's own). */
pgmg_status pgmg_dev_launch_count(pgmg_handle *h, long long *n);
/* Execution options (tuning; results do not depend on them unless noted).
 *   PGMG_OPT_GRAPHS         1 = replay each V-cycle as a captured CUDA graph (default)
 *   PGMG_OPT_CLUSTER_FIRST  first level run by the one-cluster coarse cycle
 *                           (default: the first level of <= 50000 points;
 *                           = number of levels disables it)
 *   PGMG_OPT_CLUSTER_SIZE   CTAs of that cluster: 1, 2, 4, 8, 16, or 0 (off)
 *   PGMG_OPT_SLAB_BUDGET    bytes of solution vector per z-slab of the 8-colour
 *                           sweep (default 0 = one slab).  This one
 *                           changes the update order, so results change at
 *                           rounding level and convergence slightly.
 *   PGMG_OPT_V_DOWN, PGMG_OPT_V_UP, PGMG_OPT_V_BOTTOM
 *                           the reference's public sweep counts (multigrid.hh:
 *                           122-128; defaults 2, 2, 20): level l gets v_down+l
 *                           pre- and v_up+l-1 post-sweeps (multigrid.cc:92,102).
 *   PGMG_OPT_PDL            1 = launch the V-cycle's kernels as programmatic
 *                           dependent launches, so that each is scheduled while
 *                           the one before it drains (default); 0 = plain
 *                           launches.  No counterpart in the reference.
 *   PGMG_OPT_GS_VECTOR      1 = the 8-colour sweep kernel updates 2 (FP64) or
 *                           4 (FP32) consecutive colour points per thread with
 *                           128-bit loads of their stencil coefficients; 2 = 2
 *                           points per thread (64-bit loads in FP32; as 1 in
 *                           FP64); 0 = one point per thread (default).  Only
 *                           on levels that the TMA, persistent-grid and
 *                           stencil-prefetch passes do not take.  Same
 *                           results.  No counterpart in the reference.
 *   PGMG_OPT_GS_ALTERNATE   1 = consecutive colour passes traverse the level in
 *                           opposite directions, so that each starts on the
 *                           solution planes the previous one left in L2
 *                           (default); 0 = always bottom up.  No counterpart
 *                           in the reference.
 *   PGMG_OPT_COARSE_SHARED  1 = the cluster coarse cycle sweeps a level from
 *                           shared memory: every CTA holds a copy of the
 *                           level's halo'd x and the stencils of the points
 *                           it owns, and sends each new value to the CTAs
 *                           whose points read it through distributed shared
 *                           memory (levels whose copy fits in 200 KiB;
 *                           default); 0 = x read from L2.  Same results.  No
 *                           counterpart in the reference.
 *   PGMG_OPT_GS_PREFETCH    8-colour levels of at most this many points load
 *                           each colour pass's stencil coefficients before
 *                           waiting for the previous kernel (with PGMG_OPT_PDL,
 *                           so that the loads overlap that kernel's drain);
 *                           0 = no level.  Default 4194304.  Levels that
 *                           PGMG_OPT_GS_TMA or PGMG_OPT_GRID_MAX sweep keep
 *                           those paths.  No counterpart in the reference.
 *   PGMG_OPT_INNER_DIGITS   mixed precision, adaptive schedule: the FP32
 *                           V-cycles of one refinement step are asked for at
 *                           most a 10^-d predicted reduction (1..7, default 5;
 *                           d+1 while the solve gains more than a digit per
 *                           cycle).  Changes the iterates (not the tolerance
 *                           reached).
 *   PGMG_OPT_GS_BLOCK       threads per block of the 8-colour sweep kernel:
 *                           128, 256 (default) or 512.  No counterpart in the
 *                           reference.
 *   PGMG_OPT_GRID_MAX       8-colour levels of at most this many points (and
 *                           above the cluster levels) sweep each V-cycle leg in
 *                           one persistent whole-GPU launch whose colour passes
 *                           are separated by a grid barrier with a bounded wait
 *                           (a wait that runs out makes the solve return
 *                           PGMG_ERR_TIMEOUT); 0 = off (default).  No
 *                           counterpart in the reference.
 *   PGMG_OPT_FUSED_RESTRICT 1 = the restriction of a non-periodic level
 *                           computes the fine residuals inside the restriction
 *                           kernel (tiles of the residual in shared memory, no
 *                           residual array in device memory); 0 = a residual
 *                           pass, then the restriction (default: faster on a
 *                           B200).  Same results bit for bit.
 *   PGMG_OPT_LU_WINDOW      1 (default) = the coarsest level's LU
 *                           factorisation keeps its active band window in
 *                           shared memory (where it fits in 220 KiB and the
 *                           bandwidth is at most 128); 0 = one thread block on
 *                           the dense matrix in device memory.  Same factors
 *                           bit for bit.  Takes effect at the next set-up.
 *   PGMG_OPT_GS_TMA         8-colour levels of at most this many points (one
 *                           slab, non-periodic) stage each colour pass's
 *                           stencil coefficients and sources in shared memory
 *                           with bulk copies of the Tensor Memory Accelerator,
 *                           the stencils fetched before the pass waits for the
 *                           previous kernel; 0 = off (default).  Same results
 *                           bit for bit.  No counterpart in the reference.
 *   PGMG_OPT_RAT_TILE       1 = the Galerkin operators of non-periodic coarse
 *                           levels of more than 20 000 points are built one
 *                           thread per (coarse point, stencil slot) over
 *                           shared-memory tiles; 0 = one thread per coarse
 *                           point (default: faster on a B200).  Same
 *                           operators bit for bit.  Takes effect at the next
 *                           set-up.
 *   PGMG_OPT_GS_L2_PREFETCH 8-colour levels of at most this many points (that
 *                           PGMG_OPT_GS_PREFETCH covers) prefetch the next
 *                           colour pass's stencils and sources into L2 with
 *                           bulk prefetches at the start of each pass; 0 =
 *                           off (default).  Same results.  No counterpart in
 *                           the reference.
 *   PGMG_OPT_GS_BLOCK_LEVELS threads per block of the colour sweep per level:
 *                           2 bits per level 1..15 (level l at bits 2l-2 and
 *                           2l-1): 0 = PGMG_OPT_GS_BLOCK (default), 1, 2, 3 =
 *                           128, 256, 512.  Same results.  No counterpart in
 *                           the reference.
 *   PGMG_OPT_LU_INVERSE_BAND 1 (default) = the explicit coarse inverse is
 *                           computed one warp per column over the factors'
 *                           band (where it is at most 256 rows on either side
 *                           of the diagonal); 0 = one block per column over
 *                           the dense factors.  Same inverse bit for bit.
 *                           Takes effect at the next set-up. */
enum {
    PGMG_OPT_GRAPHS = 1,
    PGMG_OPT_CLUSTER_FIRST = 2,
    PGMG_OPT_CLUSTER_SIZE = 3,
    PGMG_OPT_SLAB_BUDGET = 4,
    PGMG_OPT_V_DOWN = 5,
    PGMG_OPT_V_UP = 6,
    PGMG_OPT_V_BOTTOM = 7,
    PGMG_OPT_PDL = 8,
    PGMG_OPT_GS_BLOCK = 9,
    PGMG_OPT_GRID_MAX = 10,
    PGMG_OPT_CHECK_EVERY = 11,
    PGMG_OPT_GS_VECTOR = 12,
    PGMG_OPT_INNER_DIGITS = 13,
    PGMG_OPT_GS_ALTERNATE = 14,
    PGMG_OPT_GS_PREFETCH = 15,
    PGMG_OPT_COARSE_SHARED = 16,
    PGMG_OPT_FUSED_RESTRICT = 17,
    PGMG_OPT_LU_WINDOW = 18,
    PGMG_OPT_GS_TMA = 19,
    PGMG_OPT_RAT_TILE = 20,
    PGMG_OPT_GS_L2_PREFETCH = 21,
    PGMG_OPT_LU_INVERSE_BAND = 22,
    PGMG_OPT_GS_BLOCK_LEVELS = 23
};
pgmg_status pgmg_dev_set_option(pgmg_handle *h, int key, long long value);
/* Autotuner (no counterpart in the reference).  Times `reps` V-cycles (after
 * one untimed) of this handle's problem under candidate values of the
 * options that change no result -- PGMG_OPT_GS_BLOCK, PGMG_OPT_CLUSTER_FIRST,
 * PGMG_OPT_GS_ALTERNATE, PGMG_OPT_GS_PREFETCH, PGMG_OPT_GS_VECTOR, PGMG_OPT_CLUSTER_SIZE,
 * PGMG_OPT_GRID_MAX, PGMG_OPT_PDL, PGMG_OPT_FUSED_RESTRICT, PGMG_OPT_GS_TMA,
 * PGMG_OPT_GS_L2_PREFETCH, PGMG_OPT_GS_BLOCK_LEVELS --
 * one at a time from the best so
 * far, and keeps the fastest.  The level-0 solution is saved and restored.
 * The choice is remembered for the process per (grid, periodic axes,
 * precision, smoother, device): a later handle of the same shape takes it
 * without timing.  *ms (may be NULL): the chosen V-cycle time.  Needs
 * pgmg_dev_build_rat; synchronises. */
pgmg_status pgmg_dev_autotune(pgmg_handle *h, int reps, double *ms);
/* Self-check of the persistent sweep kernel's bounded grid barrier (no
 * counterpart in the reference): one FP64 8-colour sweep of `level` in one
 * cooperative launch; with run_out != 0 the barrier waits for one block more
 * than the launch has, so its wait runs out (about a second) and the call
 * returns PGMG_ERR_TIMEOUT with the device usable; otherwise PGMG_OK. */
pgmg_status pgmg_dev_grid_check(pgmg_handle *h, int level, int run_out);
/* Self-check of the TMA colour pass's bounded mbarrier wait (no counterpart
 * in the reference): one FP64 colour pass (the first colour) of `level`
 * with k_gs_colour_tma; with run_out != 0 every CTA's barrier expects 16
 * bytes more than its copies bring, so its wait runs out (about half a
 * second, twice) and the call returns PGMG_ERR_TIMEOUT with the device
 * usable; otherwise PGMG_OK. */
pgmg_status pgmg_dev_tma_check(pgmg_handle *h, int level, int run_out);
/* V-cycle profile (no counterpart in the reference): runs one V-cycle of the
 * handle's options, each stage launched on its own (no graph), with CUDA
 * events on the handle's stream between the stages, and writes the stage
 * times in milliseconds: ms[4*l+0] the pre-smoothing sweeps of level l,
 * ms[4*l+1] the residual and restriction from level l to l+1, ms[4*l+2] the
 * interpolation from l+1 back to l, ms[4*l+3] the post-smoothing of level l,
 * for the levels above the coarse part, and ms[4*16] the coarse part (the
 * one-cluster tail or the bottom solve); nms >= 65 entries, unused ones 0.
 * fp32 != 0 profiles the FP32 V-cycle of a PGMG_MIXED handle (its
 * correction is left in the FP32 solution; the FP64 solution is untouched).
 * *first_coarse: the first level of the coarse part.  Synchronises. */
pgmg_status pgmg_dev_profile_vcycle(pgmg_handle *h, int fp32, double *ms, int nms, int *first_coarse);
pgmg_status pgmg_dev_get_option(pgmg_handle *h, int key, long long *value);
/* Default smoother of pgmg_dev_vcycle and the solves. */
pgmg_status pgmg_dev_set_smoother(pgmg_handle *h, int smoother);
/* Number of levels (multigrid::mlevels, multigrid.hh:135) and a level's
 * size (region::m,n,o, region.hh:30-34). */
pgmg_status pgmg_dev_num_levels(pgmg_handle *h, int *nlevels);
pgmg_status pgmg_dev_level_dims(pgmg_handle *h, int level, int *mno);
/* Device bytes held by the handle. */
pgmg_status pgmg_dev_memory(pgmg_handle *h, size_t *bytes);
/* Device bytes a handle with these dims would hold (admission planning). */
pgmg_status pgmg_dev_plan_bytes(const pgmg_dims *dims, size_t *bytes);

/* ---- operator set-up -------------------------------------------------- */

/* Level-0 stencils, natural order, 27 slots per point; S6 (6 ints per point)
 * may be NULL (then every box is taken as the full 27-point box, which only
 * affects pgmg_dev_get_boxes).  Replaces region::setup_matrices
 * (region.hh:96-101) and the top-level constructor's box pass
 * (region.hh:492-519). */
pgmg_status pgmg_dev_upload_level0(pgmg_handle *h, const double *coef27, const int *S6);
/* Level-0 Q1 FEM stencils of -div(kappa grad u) assembled on the device from
 * a cell field ((m-1)(n-1)(o-1) doubles, natural order, host or device):
 * kappa itself (from_log = 0; NULL = constant 1) or g with kappa =
 * exp(sigma*g) (from_log = 1).  Same stencils, boxes and Dirichlet fix rows
 * as pgmg_problem_q1 followed by pgmg_dev_upload_level0, with 27x less data
 * to move. */
pgmg_status pgmg_dev_assemble_q1(pgmg_handle *h, const double *cells, int from_log, double sigma);
/* Level-0 source = pgmg_problem_rhs(m, n, o, seed), generated on the device. */
pgmg_status pgmg_dev_rhs_uniform(pgmg_handle *h, uint64_t seed);
/* Galerkin coarse operators A_c = (1/8) P^T A_f P on the device for every
 * level, the coarse boxes, and the coarsest-level LU.  Replaces
 * multigrid::compute_rats (multigrid.cc:138-152), region::fill_rat_bounds
 * (region.cc:598-623), region::compute_rats (region.cc:629-660) and
 * region::lu_decomposition (region_tr.cc:483-534). */
pgmg_status pgmg_dev_build_rat(pgmg_handle *h);
/* Whether the bottom level solves by LU (1) or by 24 sweeps (0). */
pgmg_status pgmg_dev_lu_enabled(pgmg_handle *h, int *enabled);
/* A level's stencils (27 slots per point) and boxes (6 ints per point). */
pgmg_status pgmg_dev_get_coef(pgmg_handle *h, int level, double *coef27);
pgmg_status pgmg_dev_get_boxes(pgmg_handle *h, int level, int *S6);

/* ---- fields ------------------------------------------------------------ */

/* Copy a field in or out, natural order, m*n*o doubles.  Replaces
 * region::setup_x_field / setup_r_field (region.hh:110-126) and reads of
 * reg[l]->x0 / r0.  PGMG_FIELD_RES is output only. */
pgmg_status pgmg_dev_set_field(pgmg_handle *h, int level, int field, const double *src);
pgmg_status pgmg_dev_get_field(pgmg_handle *h, int level, int field, double *dst);
/* out = A in on a level, natural order, m*n*o doubles each (region::Ax /
 * mul_A / unpadded_Ax, region.cc:1861-1912; multigrid.hh:226-234); on a
 * periodic axis neighbours wrap around, as in unpadded_Ax. */
pgmg_status pgmg_dev_apply(pgmg_handle *h, int level, const double *in, double *out);
/* PCG helpers of the reference's single-process path, computed on the
 * device (deterministic reductions: the same value on every call):
 *   pgmg_dev_source_soln_dot  *out = sum x*r     (region::source_soln_dot,
 *                             region.cc:1921-1931; multigrid.hh:240-242)
 *   pgmg_dev_soln_diff        *out = sum (ext_x - x)^2, ext_x natural order,
 *                             host or device (region::soln_diff,
 *                             region.hh:226-236; multigrid.hh:249-251)
 *   pgmg_dev_l0_error         *out = max |r - A x| (region::l0_error_all,
 *                             region.cc:1492-1506), bit for bit the reference's
 *   pgmg_dev_copy_r_to_x      x = r (region::copy_rhs_to_soln, region.cc:1935-1942)
 * The sums add the same terms as the reference in another order (1e-12
 * relative agreement). */
pgmg_status pgmg_dev_source_soln_dot(pgmg_handle *h, int level, double *out);
pgmg_status pgmg_dev_soln_diff(pgmg_handle *h, int level, const double *ext_x, double *out);
pgmg_status pgmg_dev_l0_error(pgmg_handle *h, int level, double *out);
pgmg_status pgmg_dev_copy_r_to_x(pgmg_handle *h, int level);
/* x = 0 on a level (region::clear_x_field, region.cc:1679-1682). */
pgmg_status pgmg_dev_clear_x(pgmg_handle *h, int level);
/* Analytic test fields (region::setup_test, region.cc:1812-1826). */
pgmg_status pgmg_dev_setup_test(pgmg_handle *h, int level, int ca, int xfield);

/* ---- hot path --------------------------------------------------------- */

/* One Gauss-Seidel sweep on a level; mode != 0 adds the backward sweep
 * (region::gauss_seidel, region.cc:355-542; multigrid::gauss_seidel,
 * multigrid.cc:180-182). */
pgmg_status pgmg_dev_gs(pgmg_handle *h, int level, int mode, int smoother);
/* Residual restriction into a level from its parent, then clear that
 * level's x (multigrid::restriction, multigrid.cc:211-224;
 * region::restriction, region.cc:546-572). */
pgmg_status pgmg_dev_restrict(pgmg_handle *h, int level);
/* Trilinear interpolation of a level's x added into its parent's x
 * (multigrid::interpolation, multigrid.cc:196-206; region.cc:576-593). */
pgmg_status pgmg_dev_interp(pgmg_handle *h, int level);
/* Coarsest-level solve (multigrid::solve_exact, multigrid.hh:265-267;
 * region::solve_exact, region_tr.cc:540-558). */
pgmg_status pgmg_dev_coarse_solve(pgmg_handle *h);
/* One V-cycle (multigrid::v_cycle, multigrid.cc:88-106): v_down+l pre- and
 * v_up+l-1 post-sweeps on level l (2 and 2 unless set with
 * pgmg_dev_set_option), coarse solve at the bottom.  smoother < 0 uses
 * the handle's default. */
pgmg_status pgmg_dev_vcycle(pgmg_handle *h, int mode, int smoother);
/* Full multigrid cycle (multigrid::fmg_cycle, multigrid.cc:109-134). */
pgmg_status pgmg_dev_fmg_cycle(pgmg_handle *h, int smoother);
/* Sum of squared residuals and of squared sources on a level (no sqrt):
 * region::l2_error_all (region.cc:1475-1490) and region::rhs_l2norm
 * (region.cc:1549-1558).  Either output may be NULL. */
pgmg_status pgmg_dev_norms(pgmg_handle *h, int level, double *res2, double *rhs2);

/* Allocation-free residual norms.  No counterpart in the reference: this is
 * for callers that cannot allocate device memory -- code under a host
 * framework that owns all of the card's memory through its own pool, or a
 * latency-critical loop where a cudaMalloc/cudaFree would stall or
 * synchronise the device.  Given caller-owned device arrays of an m x n x o
 * grid (natural order: coef27 with 27 slots per point, slot
 * (di+1)+3(dj+1)+9(dk+1); x and r with one value per point) it writes
 * out[0] = sum (r - A x)^2 and out[1] = sum r^2 (out: 2 device doubles),
 * asynchronously on `stream` (NULL = the default stream); read out after the
 * stream has finished.  It allocates nothing: its partial sums live in a
 * fixed 1 MiB array inside this library that every GPU loading it holds until
 * the process exits, so m*n*o is limited to 16,777,216 points (PGMG_ERR_ARG
 * beyond that, and for host pointers).  The first call in each CUDA context
 * (a device's primary context, or another context the caller has made
 * current) looks up that array's device address in that context; make that
 * first call before any stream capture.  All calls on a device share the
 * array (each overwrites every
 * partial sum it reads, so nothing has to be cleared): calls that overlap on
 * the GPU race and must be serialised by the caller. */
pgmg_status pgmg_residual_norms_noalloc(int m, int n, int o, const double *coef27, const double *x,
                                        const double *r, double *out, void *stream);

/* ---- solves ----------------------------------------------------------- */

/* multigrid::solve_v_cycles (multigrid.hh:182-219) with its mg_guide:
 * guide.set_tol(p_scale) is applied on the first call (p_scale > 0).
 * *result = 0 converged, 1 cycle cap, 2 NaN, as the reference returns;
 * *res2 the final squared residual; *cycles the V-cycles run. */
pgmg_status pgmg_dev_solve_v_cycles(pgmg_handle *h, double p_scale, int *result,
                                    double *res2, int *cycles);
/* Relative-residual solve: V-cycles from the current x until
 * sqrt(sum r^2 / sum b^2) < tol or max_cycles.  PGMG_MIXED handles run FP64
 * iterative refinement around FP32 V-cycles: each step computes the FP64
 * residual (and checks it), solves for the correction with FP32 V-cycles from
 * zero, and adds it in FP64.  check_every: residual check period in cycles
 * (>= 1; in mixed precision the FP32 V-cycles per refinement step), or 0 for
 * an adaptive schedule that predicts the remaining cycles from the observed
 * reduction factor (mixed precision: up to 16 cycles per step, and no more
 * than a 1e-5 predicted reduction, 1e-6 while the solve gains more than a
 * digit per cycle).  Outputs may be NULL. */
pgmg_status pgmg_dev_solve_relres(pgmg_handle *h, double tol, int max_cycles, int check_every,
                                  int *cycles, double *relres);
/* The whole solve from caller arrays (no counterpart in the reference): the
 * level-0 source r (natural order) is uploaded, x set to zero, the solve run
 * as pgmg_dev_solve_relres, and the solution written to x (natural order).
 * The same iterates, cycle count and relative residual as set_field(R) +
 * clear_x + solve_relres + get_field(X).  r and x may be host (pinned or
 * pageable) or device memory; with pinned x the solution's copy overlaps the
 * final residual check (it starts at a check that may end the solve; a later
 * one replaces it if the solve continues).  Outputs may be NULL. */
pgmg_status pgmg_dev_solve_io(pgmg_handle *h, const double *r, double *x, double tol, int max_cycles,
                              int check_every, int *cycles, double *relres);

/* ---- batched solves (many independent problems per launch) ------------- */

/* A batch has slots holding set-up handles (pgmg_dev_build_rat done) of one
 * precision, 8-colour smoother and default sweep counts; problems of any
 * size mix.  pgmg_batch_solve solves every attached problem from x = 0 to its
 * relative residual tol (or max_cycles): each launch of a step covers every
 * problem still running, per-problem convergence flags live on the device,
 * and each step is one CUDA graph per batch shape.  A problem's iterates are
 * bit for bit those of pgmg_dev_solve_relres with check_every = 1.
 * cycles / relres: per slot, arrays of max_slots (may be NULL).  The results
 * stay in each handle (pgmg_dev_get_field). */
typedef struct pgmg_batch pgmg_batch;
pgmg_status pgmg_batch_create(int max_slots, int precision, int device, pgmg_batch **out);
pgmg_status pgmg_batch_destroy(pgmg_batch *b);
const char *pgmg_batch_last_error(pgmg_batch *b);
pgmg_status pgmg_batch_attach(pgmg_batch *b, int slot, pgmg_handle *h);
pgmg_status pgmg_batch_detach(pgmg_batch *b, int slot);
pgmg_status pgmg_batch_solve(pgmg_batch *b, double tol, int max_cycles, int *cycles, double *relres);
pgmg_status pgmg_batch_launch_count(pgmg_batch *b, long long *n);
/* Step-level control for continuous batching: pgmg_batch_begin starts a
 * solve from x = 0 in an attached slot (after its handle's set-up and source
 * are complete); pgmg_batch_step runs one refinement step (residual and
 * convergence check, then a V-cycle) for every running slot and returns how
 * many still run; pgmg_batch_poll reads the per-slot flags, cycle counts and
 * relative residuals (arrays of max_slots, each may be NULL).  Slots may be
 * attached, begun and detached between steps; a batch shape that persists is
 * replayed as a captured CUDA graph (pgmg_batch_set_graphs(b, 0) turns that
 * off). */
pgmg_status pgmg_batch_begin(pgmg_batch *b, int slot);
pgmg_status pgmg_batch_step(pgmg_batch *b, double tol, int max_cycles, int *n_active);
pgmg_status pgmg_batch_poll(pgmg_batch *b, int *active, int *cycles, double *relres);
pgmg_status pgmg_batch_set_graphs(pgmg_batch *b, int on);
/* PGMG_OPT_GRAPHS and PGMG_OPT_PDL for the batch's step launches, and
 * PGMG_OPT_CHECK_EVERY: the residual-check period of every problem in cycles
 * (default 1, each problem's iterates those of pgmg_dev_solve_relres with
 * check_every = 1), or 0 for the adaptive schedule of pgmg_dev_solve_relres
 * (in mixed precision the FP32 V-cycles between checks form one refinement
 * step), evaluated per problem on the device; PGMG_OPT_CLUSTER_SIZE: CTAs of
 * each problem's coarse-tail cluster (1, 2, 4, 8 or 16; default 4, so that
 * many problems' tails run at once), or 0 for the attached handles' size
 * (which must then agree).  Results do not depend on it. */
pgmg_status pgmg_batch_set_option(pgmg_batch *b, int key, long long value);

/* ---- host problem generators (no GPU needed) ---------------------------- */

/* Cell-centred kappa = exp(sigma*g), g a seeded Gaussian field smoothed by a
 * Gaussian of `width` cells (0 = no smoothing) and normalised to zero mean,
 * unit variance; (m-1)(n-1)(o-1) cells, natural order. */
int pgmg_problem_kappa(int m, int n, int o, double sigma, uint64_t seed, double width, double *kappa);
/* Q1 trilinear FEM stencils of -div(kappa grad u) (kappa NULL = 1) with
 * Dirichlet fix rows on the boundary; fills coef27 and, if non-NULL, S6. */
int pgmg_problem_q1(int m, int n, int o, const double *kappa, double *coef27, int *S6);
/* The normalised smoothed Gaussian field g of pgmg_problem_kappa (kappa =
 * exp(sigma*g)), cells natural order. */
int pgmg_problem_gauss(int m, int n, int o, uint64_t seed, double width, double *g);
/* Right-hand side: interior nodes uniform[-1,1] from the seed, boundary 0. */
int pgmg_problem_rhs(int m, int n, int o, uint64_t seed, double *r);

#ifdef __cplusplus
}
#endif

#endif /* PGMG_DEV_H */
