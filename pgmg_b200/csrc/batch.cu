// Batched solves: many independent problems (uneven sizes) per launch.
//
// Problems are ordinary handles (their own arenas, operators built by
// pgmg_dev_build_rat) attached to the slots of a batch.  Every launch of a
// batched V-cycle covers all active problems that take part in that step:
// a per-launch block map (the "tile table": slot, first block) assigns each
// thread block to one problem, and the kernel reads that problem's level
// geometry and buffers from a device slot table.  The per-point arithmetic is
// the same device code as the single-problem kernels, so a problem's iterates
// are bit for bit the same alone and in any mix.
//
// One step of the batched solve, captured once as a CUDA graph per batch
// shape (set of slots):
//   residual of the current x for every active problem (FP64; stored FP32 as
//   the correction's source in mixed precision) and its norms ->
//   per-problem reduction that updates the problem's active flag on the
//   device (converged, or out of cycles) -> V-cycle (grid kernels on the fine
//   levels of every problem, then one cluster per problem for its coarse
//   tail) -> FP64 update.
// Finished problems drop out of later steps by their flags; the host only
// reads the flags back between steps.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <vector>

#include "handle.cuh"

using namespace pgmg;

namespace {

constexpr int kMaxSlots = 256;

// Level data of one problem, all levels.
template <class T>
struct BSlot {
    int nl, top;  // levels; first level of the cluster tail
    LevelGeom g[kMaxLv];
    T* A[kMaxLv];
    T* x[kMaxLv];
    T* r[kMaxLv];
    T* res[kMaxLv];
    const double* A64;  // level 0, FP64 (refinement residual)
    double* x64;
    const double* r64;
    double* partials;   // the handle's reduction scratch
};

// Block map of one launch: entries (slot, first block), start[n] = total.
struct BMap {
    int n;
    int slot[kMaxSlots];
    int start[kMaxSlots + 1];
};

__device__ __forceinline__ int map_entry(const BMap* __restrict__ M, int b) {
    int lo = 0, hi = M->n;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (M->start[mid] <= b) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <class T>
__global__ void __launch_bounds__(kBlock) kb_gs_colour(const BSlot<T>* __restrict__ S, const BMap* __restrict__ M,
                                                       const int* __restrict__ active, int lev, int col, int rev) {
    pdl_enter();
    // rev: walk the blocks in reverse, so that consecutive colour passes
    // alternate direction and each starts on data the previous one left in L2.
    int bi = rev ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
    int e = map_entry(M, bi);
    int s = M->slot[e];
    if (!active[s]) return;
    const BSlot<T>& B = S[s];
    long p = (long)(bi - M->start[e]) * blockDim.x + threadIdx.x;
    const LevelGeom& g = B.g[lev];
    if (p >= (long)g.M2 * g.N2 * g.O2) return;
    gs_colour_at<T>(g, B.x[lev], B.r[lev], B.A[lev], col, p);
}

// Residual of level `lev` into its scratch (restriction); blocks per problem
// = 8 colours x blocks per colour.
template <class T>
__global__ void __launch_bounds__(kBlock) kb_residual(const BSlot<T>* __restrict__ S, const BMap* __restrict__ M,
                                                      const int* __restrict__ active, int lev) {
    pdl_enter();
    int e = map_entry(M, blockIdx.x);
    int s = M->slot[e];
    if (!active[s]) return;
    const BSlot<T>& B = S[s];
    const LevelGeom& g = B.g[lev];
    long nb = nblk((long)g.M2 * g.N2 * g.O2);
    long lb = blockIdx.x - M->start[e];
    int col = (int)(lb / nb);
    double a = 0, b = 0;
    residual_at<T, T>(g, B.x[lev], B.r[lev], B.A[lev], B.res[lev], col, (lb % nb) * blockDim.x + threadIdx.x, a, b);
}

template <class T>
__global__ void __launch_bounds__(kBlock) kb_restrict(const BSlot<T>* __restrict__ S, const BMap* __restrict__ M,
                                                      const int* __restrict__ active, int lc) {
    pdl_enter();
    int e = map_entry(M, blockIdx.x);
    int s = M->slot[e];
    if (!active[s]) return;
    const BSlot<T>& B = S[s];
    long q = (long)(blockIdx.x - M->start[e]) * blockDim.x + threadIdx.x;
    restrict_fast_at<T>(B.g[lc - 1], B.g[lc], B.res[lc - 1], B.r[lc], B.x[lc], q);
}

template <class T>
__global__ void __launch_bounds__(kBlock) kb_interp(const BSlot<T>* __restrict__ S, const BMap* __restrict__ M,
                                                    const int* __restrict__ active, int lc) {
    pdl_enter();
    int e = map_entry(M, blockIdx.x);
    int s = M->slot[e];
    if (!active[s]) return;
    const BSlot<T>& B = S[s];
    long q = (long)(blockIdx.x - M->start[e]) * blockDim.x + threadIdx.x;
    interp_cube_at<T>(B.g[lc - 1], B.g[lc], B.x[lc - 1], B.x[lc], q);  // q: a cube of level lc-1
}

// FP64 residual of level 0 (or the source alone when x = 0) with the same
// per-problem block structure and partial layout as k_residual / k_source;
// stores it as the FP32 correction source when TO = float.
template <class T, class TO>
__global__ void __launch_bounds__(kBlock) kb_check(const BSlot<T>* __restrict__ S, const BMap* __restrict__ M,
                                                   const int* __restrict__ active, const int* __restrict__ first,
                                                   const int* __restrict__ due) {
    pdl_enter();
    __shared__ double sh[64];
    int e = map_entry(M, blockIdx.x);
    int s = M->slot[e];
    if (!active[s] || !due[s]) return;
    const BSlot<T>& B = S[s];
    const LevelGeom& g = B.g[0];
    long nc = (long)g.M2 * g.N2 * g.O2;
    long nb = nblk(nc);
    long lb = blockIdx.x - M->start[e];
    int col = (int)(lb / nb);
    long p = (lb % nb) * blockDim.x + threadIdx.x;
    TO* out = std::is_same<TO, float>::value ? reinterpret_cast<TO*>(B.r[0]) : nullptr;
    double a = 0, b = 0;
    if (first[s]) {
        if (p < nc) {
            double rv = B.r64[(long)col * g.Nc + p];
            if (out) out[(long)col * g.Nc + p] = (TO)rv;
            a = rv * rv;
        }
        b = a;
    } else {
        residual_at<double, TO>(g, B.x64, B.r64, B.A64, out, col, p, a, b);
    }
    block_sum2(a, b, sh);
    if (threadIdx.x == 0) {
        B.partials[2 * lb] = a;
        B.partials[2 * lb + 1] = b;
    }
}

// Per-problem residual-check schedule, on the device: the cycle of the next
// check and the history the prediction uses (pgmg_dev_solve_relres's
// CheckPlan, one per slot; rho0 is the mean reduction of the slot's last
// solve).
struct BPlan {
    int next, first_n, prev_n, last_n;
    double first_r, prev_r, last_r, rho0;
};

__device__ inline void bplan_reset(BPlan& P) {
    P.next = 0;
    P.first_n = P.prev_n = P.last_n = -1;
    P.first_r = P.prev_r = P.last_r = 0;
}

// Cycle of the next check after a check at cycle nc (same rules as the
// single-problem schedule).
__device__ inline int bplan_next(const BPlan& P, int every, int mixed, int nc, double tol, int max_cycles) {
    int nx;
    double q = (P.prev_n >= 0 && P.last_r > 0 && P.prev_r > 0)
                   ? pow(P.last_r / P.prev_r, 1.0 / (P.last_n - P.prev_n)) : P.rho0;
    if (every >= 1) {
        nx = nc + every;
    } else if (!(q > 0) || q >= 0.9 || !(P.last_r > 0)) {
        nx = nc + 1;
    } else {
        int n = (int)ceil(log(tol / P.last_r) / log(q));
        if (n < 1) n = 1;
        if (n > 1 && P.last_r * pow(q, n - 1) < kSlack * tol) n--;
        nx = nc + n;
        if (mixed) nx = nc + ir_inner_cycles(n, q, kInnerDigits);
    }
    if (nx > max_cycles) nx = max_cycles;
    if (nx < nc + 1) nx = nc + 1;
    return nx;
}

// One block per problem due for a check: the reduction of
// k_reduce_partials, then the convergence decision of pgmg_dev_solve_relres:
// stop when the relative residual is below tol (or NaN, or the cycle budget
// is spent), otherwise schedule the next check.
template <class T>
__global__ void __launch_bounds__(1024) kb_reduce(const BSlot<T>* __restrict__ S, const BMap* __restrict__ M,
                                                  int* __restrict__ active, int* __restrict__ first,
                                                  const int* __restrict__ cycles, double* __restrict__ relres,
                                                  BPlan* __restrict__ plans, const int* __restrict__ due,
                                                  double tol, int max_cycles, int every, int mixed) {
    pdl_enter();
    __shared__ double sh[64];
    int s = M->slot[blockIdx.x];
    if (!active[s] || !due[s]) return;
    const BSlot<T>& B = S[s];
    const LevelGeom& g = B.g[0];
    long nb = nblk((long)g.M2 * g.N2 * g.O2) * 8;
    double a = 0, b = 0;
    for (long q = threadIdx.x; q < nb; q += blockDim.x) {
        a += B.partials[2 * q];
        b += B.partials[2 * q + 1];
    }
    block_sum2(a, b, sh);
    if (threadIdx.x == 0) {
        double rr = b > 0 ? sqrt(a / b) : sqrt(a);
        relres[s] = rr;
        first[s] = 0;
        BPlan& P = plans[s];
        int nc = cycles[s];
        if (isnan(rr) || rr < tol || nc >= max_cycles) {
            active[s] = 0;
            if (nc > P.first_n && P.first_n >= 0 && P.first_r > 0 && rr > 0) {
                double q = pow(rr / P.first_r, 1.0 / (nc - P.first_n));
                if (q > 0 && q < 0.9) P.rho0 = q;
            }
        } else {
            if (P.first_n < 0) { P.first_n = nc; P.first_r = rr; }
            P.prev_n = P.last_n; P.prev_r = P.last_r; P.last_n = nc; P.last_r = rr;
            P.next = bplan_next(P, every, mixed, nc, tol, max_cycles);
        }
    }
}

// After the step's V-cycle: count it, and mark the problems whose next step
// starts with a check (their correction is complete).
__global__ void kb_advance(const BMap* __restrict__ M, const int* __restrict__ active, int* __restrict__ cycles,
                           const BPlan* __restrict__ plans, int* __restrict__ due) {
    pdl_enter();
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M->n) return;
    int s = M->slot[e];
    if (!active[s]) return;
    int c = cycles[s] + 1;
    cycles[s] = c;
    due[s] = c >= plans[s].next;
}

__global__ void __launch_bounds__(kBlock) kb_clear32(const BSlot<float>* __restrict__ S, const BMap* __restrict__ M,
                                                     const int* __restrict__ active, const int* __restrict__ due) {
    pdl_enter();
    int e = map_entry(M, blockIdx.x);
    int s = M->slot[e];
    if (!active[s] || !due[s]) return;
    const LevelGeom& g = S[s].g[0];
    long q = (long)(blockIdx.x - M->start[e]) * blockDim.x + threadIdx.x;
    if (q >= g.npts) return;
    int i, j, k;
    decode_nat(g, q, i, j, k);
    S[s].x[0][g.xi(i, j, k)] = 0.0f;
}

__global__ void __launch_bounds__(kBlock) kb_add32(const BSlot<float>* __restrict__ S, const BMap* __restrict__ M,
                                                   const int* __restrict__ active, const int* __restrict__ due) {
    pdl_enter();
    int e = map_entry(M, blockIdx.x);
    int s = M->slot[e];
    if (!active[s] || !due[s]) return;
    const LevelGeom& g = S[s].g[0];
    long q = (long)(blockIdx.x - M->start[e]) * blockDim.x + threadIdx.x;
    if (q >= g.npts) return;
    int i, j, k;
    decode_nat(g, q, i, j, k);
    long c = g.xi(i, j, k);
    S[s].x64[c] = S[s].x64[c] + (double)S[s].x[0][c];
}

__global__ void __launch_bounds__(kBlock) kb_clear64(const BSlot<double>* S64, const BSlot<float>* S32,
                                                     const BMap* __restrict__ M) {
    int e = map_entry(M, blockIdx.x);
    int s = M->slot[e];
    const LevelGeom& g = S64 ? S64[s].g[0] : S32[s].g[0];
    double* x64 = S64 ? S64[s].x64 : S32[s].x64;
    long q = (long)(blockIdx.x - M->start[e]) * blockDim.x + threadIdx.x;
    if (q >= g.npts) return;
    int i, j, k;
    decode_nat(g, q, i, j, k);
    x64[g.xi(i, j, k)] = 0.0;
}

__global__ void kb_reset(const BMap* __restrict__ M, int* active, int* first, int* cycles, double* relres,
                         BPlan* plans, int* due, const double* __restrict__ rho0) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M->n) return;
    int s = M->slot[e];
    active[s] = 1;
    first[s] = 1;
    cycles[s] = 0;
    relres[s] = 0;
    due[s] = 1;
    bplan_reset(plans[s]);
    plans[s].rho0 = rho0[s];
}

// Starts one slot: x = 0 on its level 0 and fresh flags; rho0 is the
// problem's remembered reduction factor.
__global__ void __launch_bounds__(kBlock) kb_begin(LevelGeom g, double* x64, int s, int* active, int* first,
                                                   int* cycles, double* relres, BPlan* plans, int* due,
                                                   double rho0) {
    long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q == 0) {
        active[s] = 1;
        first[s] = 1;
        cycles[s] = 0;
        relres[s] = 0;
        due[s] = 1;
        bplan_reset(plans[s]);
        plans[s].rho0 = rho0;
    }
    if (q >= g.npts) return;
    int i, j, k;
    decode_nat(g, q, i, j, k);
    x64[g.xi(i, j, k)] = 0.0;
}

}  // namespace

struct pgmg_batch {
    int precision = PGMG_MIXED;
    int device = 0;
    // CTAs of each problem's coarse-tail cluster.  Batches hold many small
    // problems, whose tails run side by side: 4-CTA clusters let four times
    // as many run at once as the single-problem 16 and were fastest on the
    // 96-problem workload.  PGMG_OPT_CLUSTER_SIZE 0 follows the handles.
    int csize = 4;
    bool csize_fixed = true;
    cudaStream_t stream = nullptr;
    std::vector<pgmg_handle*> slots;  // nullptr = free
    // device memory
    void* slot_table = nullptr;  // BSlot<T>[kMaxSlots]
    void* plan_table = nullptr;  // CoarsePlan<T>[kMaxSlots]
    BMap* maps = nullptr;        // built per shape
    int nmaps_cap = 0;
    int* active = nullptr;
    int* first = nullptr;
    int* cycles = nullptr;
    double* relres = nullptr;
    BPlan* plans = nullptr;  // residual-check schedule per slot
    double* rho_in = nullptr;  // per-slot starting reduction factors (staging)
    int* due = nullptr;      // 1: the slot's next step starts with a check
    int* cluster_slots = nullptr;
    // shape
    bool dirty = true;
    std::vector<int> members;  // occupied slots, ascending
    int maxtop = 0, maxnl = 0;
    std::vector<BMap> hmaps;
    int map_gs[kMaxLv], map_res[kMaxLv], map_rst[kMaxLv], map_int[kMaxLv], map_chk = -1, map_pt0 = -1, map_red = -1;
    int v_down = 2, v_up = 2;
    cudaGraphExec_t step_graph[2] = {nullptr, nullptr};  // one captured step (index 0 used)
    int stable_steps = 0;  // steps run since the last shape change (capture from the second)
    long long graph_nodes = 0;  // kernels in the captured step
    bool use_graphs = true;
    bool pdl = true;  // step kernels as programmatic dependent launches
    double cap_tol = -1;  // tol and cycle cap the step graphs were captured with
    int cap_max = -1;
    int check_every = 1;  // residual check period in cycles, 0 = adaptive
    long long launches = 0;
    char err[512] = {0};
};

namespace {

pgmg_status bfail(pgmg_batch* b, pgmg_status st, const char* fmt, ...) {
    if (b) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(b->err, sizeof(b->err), fmt, ap);
        va_end(ap);
    }
    return st;
}

#define BCK(call)                                                                                       \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return bfail(b, PGMG_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)
#define BTRY(expr)                     \
    do {                               \
        pgmg_status s_ = (expr);       \
        if (s_ != PGMG_OK) return s_;  \
    } while (0)

void drop_step_graphs(pgmg_batch* b) {
    for (auto& g : b->step_graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

template <class T>
void fill_slot(pgmg_handle* h, BSlot<T>& B) {
    B.nl = h->nl;
    B.top = h->coarse_first;
    for (int l = 0; l < h->nl; l++) {
        View<T> v = std::is_same<T, float>::value ? View<T>{(T*)h->L[l].A32, (T*)h->L[l].x32, (T*)h->L[l].r32,
                                                             (T*)h->L[l].res32}
                                                   : View<T>{(T*)h->L[l].A64, (T*)h->L[l].x64, (T*)h->L[l].r64,
                                                             (T*)h->L[l].res64};
        B.g[l] = h->L[l].g;
        B.A[l] = v.A; B.x[l] = v.x; B.r[l] = v.r; B.res[l] = v.res;
    }
    B.A64 = h->L[0].A64;
    B.x64 = h->L[0].x64;
    B.r64 = h->L[0].r64;
    B.partials = h->partials;
}

int add_map(pgmg_batch* b, const std::vector<std::pair<int, long>>& entries) {
    BMap M;
    M.n = (int)entries.size();
    long tot = 0;
    for (int e = 0; e < M.n; e++) {
        M.slot[e] = entries[e].first;
        M.start[e] = (int)tot;
        tot += entries[e].second;
    }
    M.start[M.n] = (int)tot;
    b->hmaps.push_back(M);
    return (int)b->hmaps.size() - 1;
}

inline int map_blocks(const pgmg_batch* b, int m) { return b->hmaps[m].start[b->hmaps[m].n]; }

// Builds slot tables, plans and block maps for the current members.
template <class T>
pgmg_status build_shape(pgmg_batch* b) {
    b->members.clear();
    for (int s = 0; s < (int)b->slots.size(); s++)
        if (b->slots[s]) b->members.push_back(s);
    std::vector<BSlot<T>> tab(kMaxSlots);
    std::vector<CoarsePlan<T>> plans(kMaxSlots);
    b->maxtop = 0;
    b->maxnl = 0;
    for (int s : b->members) {
        pgmg_handle* h = b->slots[s];
        fill_slot<T>(h, tab[s]);
        CoarsePlan<T>& P = plans[s];
        P.first = h->coarse_first;
        P.nl = h->nl;
        P.lu_ok = h->lu_ok;
        P.slab_budget = 0;
        P.v_down = b->v_down;
        P.v_up = b->v_up;
        P.Minv = h->Minv;
        for (int l = 0; l < h->nl; l++) {
            P.g[l] = tab[s].g[l];
            P.A[l] = tab[s].A[l]; P.x[l] = tab[s].x[l]; P.r[l] = tab[s].r[l]; P.res[l] = tab[s].res[l];
        }
        if (h->coarse_first > b->maxtop) b->maxtop = h->coarse_first;
        if (h->nl > b->maxnl) b->maxnl = h->nl;
    }
    b->hmaps.clear();
    for (int l = 0; l < kMaxLv; l++) b->map_gs[l] = b->map_res[l] = b->map_rst[l] = b->map_int[l] = -1;
    for (int l = 0; l < b->maxtop; l++) {
        std::vector<std::pair<int, long>> gs, res, rst, itp;
        for (int s : b->members) {
            pgmg_handle* h = b->slots[s];
            if (l >= h->coarse_first) continue;
            const LevelGeom& g = h->L[l].g;
            long nc = (long)g.M2 * g.N2 * g.O2;
            gs.push_back({s, nblk(nc)});
            res.push_back({s, 8 * nblk(nc)});
            rst.push_back({s, nblk(h->L[l + 1].g.npts)});
            itp.push_back({s, nblk(nc)});  // interpolation from l+1 into l, one thread per cube of l
        }
        if (gs.empty()) continue;
        b->map_gs[l] = add_map(b, gs);
        b->map_res[l] = add_map(b, res);
        b->map_rst[l + 1] = add_map(b, rst);
        b->map_int[l + 1] = add_map(b, itp);
    }
    std::vector<std::pair<int, long>> chk, pt0, red;
    std::vector<int> cl;
    for (int s : b->members) {
        const LevelGeom& g = b->slots[s]->L[0].g;
        chk.push_back({s, 8 * nblk((long)g.M2 * g.N2 * g.O2)});
        pt0.push_back({s, nblk(g.npts)});
        red.push_back({s, 1});
        cl.push_back(s);
    }
    b->map_chk = add_map(b, chk);
    b->map_pt0 = add_map(b, pt0);
    b->map_red = add_map(b, red);
    if ((int)b->hmaps.size() > b->nmaps_cap) {
        if (b->maps) cudaFree(b->maps);
        b->nmaps_cap = (int)b->hmaps.size() + 8;
        BCK(cudaMalloc(&b->maps, sizeof(BMap) * b->nmaps_cap));
    }
    BCK(cudaMemcpyAsync(b->maps, b->hmaps.data(), sizeof(BMap) * b->hmaps.size(), cudaMemcpyHostToDevice, b->stream));
    BCK(cudaMemcpyAsync(b->slot_table, tab.data(), sizeof(BSlot<T>) * kMaxSlots, cudaMemcpyHostToDevice, b->stream));
    BCK(cudaMemcpyAsync(b->plan_table, plans.data(), sizeof(CoarsePlan<T>) * kMaxSlots, cudaMemcpyHostToDevice,
                        b->stream));
    BCK(cudaMemcpyAsync(b->cluster_slots, cl.data(), sizeof(int) * cl.size(), cudaMemcpyHostToDevice, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    drop_step_graphs(b);
    b->dirty = false;
    return PGMG_OK;
}

// A step kernel (one that starts with pdl_enter()).
#define BLAUNCH(grid, block, ...)                                      \
    do {                                                               \
        b->launches++;                                                 \
        BCK(launch_k(b->stream, b->pdl, grid, block, __VA_ARGS__));    \
    } while (0)
#define BKL()                           \
    do {                                \
        b->launches++;                  \
        BCK(cudaGetLastError());        \
    } while (0)

template <class T>
pgmg_status enqueue_step(pgmg_batch* b, double tol, int max_cycles) {
    const BSlot<T>* S = static_cast<const BSlot<T>*>(b->slot_table);
    auto M = [&](int m) { return b->maps + m; };
    using TO = T;
    const int mixed = std::is_same<T, float>::value ? 1 : 0;
    BLAUNCH(map_blocks(b, b->map_chk), kBlock, kb_check<T, TO>, S, M(b->map_chk), b->active, b->first, b->due);
    BLAUNCH((int)b->members.size(), 1024, kb_reduce<T>, S, M(b->map_red), b->active, b->first, b->cycles,
            b->relres, b->plans, b->due, tol, max_cycles, b->check_every, mixed);
    if (mixed) {
        BLAUNCH(map_blocks(b, b->map_pt0), kBlock, kb_clear32, reinterpret_cast<const BSlot<float>*>(S),
                M(b->map_pt0), b->active, b->due);
    }
    for (int l = 0; l < b->maxtop; l++) {
        if (b->map_gs[l] < 0) continue;
        for (int sw = 0; sw < b->v_down + l; sw++)
            for (int c = 0; c < 8; c++) {
                BLAUNCH(map_blocks(b, b->map_gs[l]), kBlock, kb_gs_colour<T>, S, M(b->map_gs[l]), b->active, l, colour_seq(c), c & 1);
            }
        BLAUNCH(map_blocks(b, b->map_res[l]), kBlock, kb_residual<T>, S, M(b->map_res[l]), b->active, l);
        BLAUNCH(map_blocks(b, b->map_rst[l + 1]), kBlock, kb_restrict<T>, S, M(b->map_rst[l + 1]), b->active, l + 1);
    }
    {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(b->members.size() * b->csize), 1, 1);
        cfg.blockDim = dim3(kClusterThreads, 1, 1);
        cfg.stream = b->stream;
        // No dynamic shared memory: the tails sweep x from L2.  (The
        // single-problem shared-memory sweeps were slower here: a batched
        // problem's tail level gets few sweeps per call, and copying the
        // level in and staging its stencils cost more than the passes saved
        // -- 96 mixed problems, 4-CTA clusters: 76.9 ms per batch without,
        // 87.9 ms with.)
        cudaLaunchAttribute attr[2];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = b->csize;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[1].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = b->pdl ? 2 : 1;
        const CoarsePlan<T>* plans = static_cast<const CoarsePlan<T>*>(b->plan_table);
        const int* cs = b->cluster_slots;
        const int* act = b->active;
        BCK(cudaLaunchKernelEx(&cfg, k_coarse_cycle<T>, plans, cs, act, 0));
        b->launches++;
    }
    for (int l = b->maxtop; l > 0; l--) {
        if (b->map_int[l] < 0) continue;
        BLAUNCH(map_blocks(b, b->map_int[l]), kBlock, kb_interp<T>, S, M(b->map_int[l]), b->active, l);
        for (int sw = 0; sw < b->v_up + l - 1; sw++)
            for (int c = 0; c < 8; c++) {
                BLAUNCH(map_blocks(b, b->map_gs[l - 1]), kBlock, kb_gs_colour<T>, S, M(b->map_gs[l - 1]), b->active, l - 1, colour_seq(c), c & 1);
            }
    }
    int nm = (int)b->members.size();
    BLAUNCH((nm + 127) / 128, 128, kb_advance, M(b->map_red), b->active, b->cycles, b->plans, b->due);
    if (mixed) {
        BLAUNCH(map_blocks(b, b->map_pt0), kBlock, kb_add32, reinterpret_cast<const BSlot<float>*>(S),
                M(b->map_pt0), b->active, b->due);
    }
    return PGMG_OK;
}

template <class T>
pgmg_status run_step(pgmg_batch* b, double tol, int max_cycles) {
    // tol and the cycle cap are graph parameters: recapture if they change.
    if (tol != b->cap_tol || max_cycles != b->cap_max) {
        drop_step_graphs(b);
        b->cap_tol = tol;
        b->cap_max = max_cycles;
    }
    // A new shape runs its first step with plain launches; a shape that
    // persists is captured once and replayed.
    if (!b->use_graphs || b->stable_steps < 1) {
        b->stable_steps++;
        return enqueue_step<T>(b, tol, max_cycles);
    }
    cudaGraphExec_t& ex = b->step_graph[0];
    if (!ex) {
        long long before = b->launches;
        BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        pgmg_status st = enqueue_step<T>(b, tol, max_cycles);
        b->graph_nodes = b->launches - before;
        b->launches = before;
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
        if (st != PGMG_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        BCK(e);
        e = cudaGraphInstantiate(&ex, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            ex = nullptr;
            return bfail(b, PGMG_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
        }
    }
    BCK(cudaGraphLaunch(ex, b->stream));
    b->launches += b->graph_nodes;
    b->stable_steps++;
    return PGMG_OK;
}

template <class T>
pgmg_status batch_step(pgmg_batch* b, double tol, int max_cycles, int* n_active) {
    TraceRange tr("pgmg batch step");
    if (b->dirty) {
        BTRY(build_shape<T>(b));
        b->stable_steps = 0;
    }
    if (b->members.empty()) {
        if (n_active) *n_active = 0;
        return PGMG_OK;
    }
    BTRY(run_step<T>(b, tol, max_cycles));
    std::vector<int> act(kMaxSlots);
    BCK(cudaMemcpyAsync(act.data(), b->active, sizeof(int) * kMaxSlots, cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    int na = 0;
    for (int s : b->members) na += act[s] ? 1 : 0;
    if (n_active) *n_active = na;
    return PGMG_OK;
}

template <class T>
pgmg_status batch_solve(pgmg_batch* b, double tol, int max_cycles, int* cycles, double* relres) {
    if (b->dirty) {
        BTRY(build_shape<T>(b));
        b->stable_steps = 0;
    }
    if (b->members.empty()) return PGMG_OK;
    int nm = (int)b->members.size();
    // Each problem starts from its handle's remembered reduction factor.
    std::vector<double> rho(kMaxSlots, 0.0);
    for (int s : b->members) rho[s] = b->slots[s]->last_rho;
    BCK(cudaMemcpyAsync(b->rho_in, rho.data(), sizeof(double) * kMaxSlots, cudaMemcpyHostToDevice, b->stream));
    kb_reset<<<(nm + 127) / 128, 128, 0, b->stream>>>(b->maps + b->map_red, b->active, b->first, b->cycles, b->relres,
                                                    b->plans, b->due, b->rho_in);
    BKL();
    kb_clear64<<<map_blocks(b, b->map_pt0), kBlock, 0, b->stream>>>(
        std::is_same<T, double>::value ? static_cast<const BSlot<double>*>(b->slot_table) : nullptr,
        std::is_same<T, float>::value ? static_cast<const BSlot<float>*>(b->slot_table) : nullptr,
        b->maps + b->map_pt0);
    BKL();
    for (int s : b->members) b->slots[s]->x0_zero = false;
    for (int step = 0; step <= max_cycles; step++) {
        int na = 0;
        BTRY(batch_step<T>(b, tol, max_cycles, &na));
        if (!na) break;
    }
    std::vector<int> cyc(kMaxSlots);
    std::vector<double> rr(kMaxSlots);
    std::vector<BPlan> pl(kMaxSlots);
    BCK(cudaMemcpyAsync(cyc.data(), b->cycles, sizeof(int) * kMaxSlots, cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaMemcpyAsync(rr.data(), b->relres, sizeof(double) * kMaxSlots, cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaMemcpyAsync(pl.data(), b->plans, sizeof(BPlan) * kMaxSlots, cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    for (int s : b->members) b->slots[s]->last_rho = pl[s].rho0;  // learned, for the problem's next solve
    for (int s = 0; s < (int)b->slots.size(); s++) {
        if (cycles) cycles[s] = b->slots[s] ? cyc[s] : 0;
        if (relres) relres[s] = b->slots[s] ? rr[s] : 0;
    }
    return PGMG_OK;
}

}  // namespace

extern "C" {

pgmg_status pgmg_batch_create(int max_slots, int precision, int device, pgmg_batch** out) {
    if (!out || max_slots < 1 || max_slots > kMaxSlots) return PGMG_ERR_ARG;
    if (precision != PGMG_FP64 && precision != PGMG_MIXED) return PGMG_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return PGMG_ERR_NO_DEVICE;
    }
    pgmg_batch* b = new pgmg_batch;
    b->precision = precision;
    if (device >= 0) cudaSetDevice(device);
    cudaGetDevice(&b->device);
    b->slots.assign(max_slots, nullptr);
    size_t tb = precision == PGMG_MIXED ? sizeof(BSlot<float>) : sizeof(BSlot<double>);
    size_t pb = precision == PGMG_MIXED ? sizeof(CoarsePlan<float>) : sizeof(CoarsePlan<double>);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&b->slot_table, tb * kMaxSlots) != cudaSuccess ||
        cudaMalloc(&b->plan_table, pb * kMaxSlots) != cudaSuccess ||
        cudaMalloc(&b->active, sizeof(int) * kMaxSlots) != cudaSuccess ||
        cudaMalloc(&b->first, sizeof(int) * kMaxSlots) != cudaSuccess ||
        cudaMalloc(&b->cycles, sizeof(int) * kMaxSlots) != cudaSuccess ||
        cudaMalloc(&b->relres, sizeof(double) * kMaxSlots) != cudaSuccess ||
        cudaMalloc(&b->plans, sizeof(BPlan) * kMaxSlots) != cudaSuccess ||
        cudaMalloc(&b->rho_in, sizeof(double) * kMaxSlots) != cudaSuccess ||
        cudaMalloc(&b->due, sizeof(int) * kMaxSlots) != cudaSuccess ||
        cudaMalloc(&b->cluster_slots, sizeof(int) * kMaxSlots) != cudaSuccess) {
        cudaGetLastError();
        pgmg_batch_destroy(b);
        return PGMG_ERR_MEMORY;
    }
    cudaMemsetAsync(b->active, 0, sizeof(int) * kMaxSlots, b->stream);
    cudaMemsetAsync(b->first, 0, sizeof(int) * kMaxSlots, b->stream);
    cudaMemsetAsync(b->cycles, 0, sizeof(int) * kMaxSlots, b->stream);
    cudaMemsetAsync(b->plans, 0, sizeof(BPlan) * kMaxSlots, b->stream);
    cudaMemsetAsync(b->due, 0, sizeof(int) * kMaxSlots, b->stream);
    cudaStreamSynchronize(b->stream);
    *out = b;
    return PGMG_OK;
}

pgmg_status pgmg_batch_destroy(pgmg_batch* b) {
    if (!b) return PGMG_ERR_ARG;
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_step_graphs(b);
    cudaFree(b->slot_table);
    cudaFree(b->plan_table);
    cudaFree(b->maps);
    cudaFree(b->active);
    cudaFree(b->first);
    cudaFree(b->cycles);
    cudaFree(b->relres);
    cudaFree(b->plans);
    cudaFree(b->rho_in);
    cudaFree(b->due);
    cudaFree(b->cluster_slots);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return PGMG_OK;
}

const char* pgmg_batch_last_error(pgmg_batch* b) { return b ? b->err : "null batch"; }

pgmg_status pgmg_batch_attach(pgmg_batch* b, int slot, pgmg_handle* h) {
    if (!b || !h || slot < 0 || slot >= (int)b->slots.size()) return PGMG_ERR_ARG;
    if (b->slots[slot]) return bfail(b, PGMG_ERR_ARG, "slot %d is occupied", slot);
    if (!h->built) return bfail(b, PGMG_ERR_SETUP, "problem operators not built");
    if (h->dims.precision != b->precision) return bfail(b, PGMG_ERR_ARG, "precision differs from the batch's");
    if (h->prd) return bfail(b, PGMG_ERR_UNSUPPORTED, "batched problems are non-periodic");
    if (h->dims.smoother != PGMG_SMOOTH_MC8 || h->cluster_size == 0 || h->slab_budget != 0 ||
        h->dims.coarse == PGMG_COARSE_LU_EXACT)
        return bfail(b, PGMG_ERR_UNSUPPORTED, "batched problems use the 8-colour smoother with the cluster coarse cycle");
    if (h->v_down != b->v_down || h->v_up != b->v_up)
        return bfail(b, PGMG_ERR_UNSUPPORTED, "batched problems use the batch's sweep counts");
    if (h->device != b->device) return bfail(b, PGMG_ERR_ARG, "problem lives on another device");
    if (!b->csize_fixed) {
        b->csize = h->cluster_size;
        for (pgmg_handle* o : b->slots)
            if (o && o->cluster_size != b->csize) return bfail(b, PGMG_ERR_UNSUPPORTED, "cluster sizes differ");
    }
    b->slots[slot] = h;
    b->dirty = true;
    return PGMG_OK;
}

pgmg_status pgmg_batch_detach(pgmg_batch* b, int slot) {
    if (!b || slot < 0 || slot >= (int)b->slots.size()) return PGMG_ERR_ARG;
    if (b->slots[slot]) {
        // The reduction factor the slot learned goes back to its problem.
        BPlan p;
        BCK(cudaMemcpyAsync(&p, b->plans + slot, sizeof(BPlan), cudaMemcpyDeviceToHost, b->stream));
        BCK(cudaStreamSynchronize(b->stream));
        b->slots[slot]->last_rho = p.rho0;
    }
    BCK(cudaMemsetAsync(b->active + slot, 0, sizeof(int), b->stream));
    b->slots[slot] = nullptr;
    b->dirty = true;
    return PGMG_OK;
}

pgmg_status pgmg_batch_begin(pgmg_batch* b, int slot) {
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot]) return PGMG_ERR_ARG;
    pgmg_handle* h = b->slots[slot];
    BCK(cudaStreamSynchronize(h->stream));  // its set-up and source are complete
    const LevelGeom& g = h->L[0].g;
    kb_begin<<<nblk(g.npts), kBlock, 0, b->stream>>>(g, h->L[0].x64, slot, b->active, b->first, b->cycles, b->relres,
                                                     b->plans, b->due, h->last_rho);
    BKL();
    h->x0_zero = false;
    return PGMG_OK;
}

pgmg_status pgmg_batch_step(pgmg_batch* b, double tol, int max_cycles, int* n_active) {
    if (!b || max_cycles < 0) return PGMG_ERR_ARG;
    if (b->precision == PGMG_MIXED) return batch_step<float>(b, tol, max_cycles, n_active);
    return batch_step<double>(b, tol, max_cycles, n_active);
}

pgmg_status pgmg_batch_poll(pgmg_batch* b, int* active, int* cycles, double* relres) {
    if (!b) return PGMG_ERR_ARG;
    size_t ns = b->slots.size();
    if (active) BCK(cudaMemcpyAsync(active, b->active, sizeof(int) * ns, cudaMemcpyDeviceToHost, b->stream));
    if (cycles) BCK(cudaMemcpyAsync(cycles, b->cycles, sizeof(int) * ns, cudaMemcpyDeviceToHost, b->stream));
    if (relres) BCK(cudaMemcpyAsync(relres, b->relres, sizeof(double) * ns, cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    return PGMG_OK;
}

pgmg_status pgmg_batch_set_graphs(pgmg_batch* b, int on) {
    if (!b) return PGMG_ERR_ARG;
    drop_step_graphs(b);
    b->use_graphs = on != 0;
    return PGMG_OK;
}

pgmg_status pgmg_batch_set_option(pgmg_batch* b, int key, long long value) {
    if (!b) return PGMG_ERR_ARG;
    switch (key) {
        case PGMG_OPT_GRAPHS: b->use_graphs = value != 0; break;
        case PGMG_OPT_PDL: b->pdl = value != 0; break;
        case PGMG_OPT_CHECK_EVERY:
            if (value < 0) return bfail(b, PGMG_ERR_ARG, "check period must be >= 0");
            b->check_every = (int)value;
            break;
        case PGMG_OPT_CLUSTER_SIZE:
            // CTAs of each problem's coarse-tail cluster (0: the attached
            // handles' size).  Smaller clusters let more problems' tails run
            // at once.
            if (value != 0 && value != 1 && value != 2 && value != 4 && value != 8 && value != 16)
                return bfail(b, PGMG_ERR_ARG, "cluster size must be 0, 1, 2, 4, 8 or 16");
            b->csize_fixed = value != 0;
            if (value) {
                b->csize = (int)value;
            } else {
                b->csize = 0;
                for (pgmg_handle* o : b->slots)
                    if (o) {
                        if (b->csize && o->cluster_size != b->csize)
                            return bfail(b, PGMG_ERR_UNSUPPORTED, "cluster sizes differ");
                        b->csize = o->cluster_size;
                    }
            }
            break;
        default: return bfail(b, PGMG_ERR_ARG, "unknown batch option %d", key);
    }
    drop_step_graphs(b);
    return PGMG_OK;
}

pgmg_status pgmg_batch_solve(pgmg_batch* b, double tol, int max_cycles, int* cycles, double* relres) {
    if (!b || max_cycles < 0) return PGMG_ERR_ARG;
    TraceRange tr("pgmg batch solve");
    // Work of the attached handles issued on their own streams must be done.
    for (pgmg_handle* h : b->slots)
        if (h) BCK(cudaStreamSynchronize(h->stream));
    if (b->precision == PGMG_MIXED) return batch_solve<float>(b, tol, max_cycles, cycles, relres);
    return batch_solve<double>(b, tol, max_cycles, cycles, relres);
}

pgmg_status pgmg_batch_launch_count(pgmg_batch* b, long long* n) {
    if (!b || !n) return PGMG_ERR_ARG;
    *n = b->launches;
    return PGMG_OK;
}

}  // extern "C"
