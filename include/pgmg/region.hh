/* Drop-in region (reference region.hh:12-467): one level of a multigrid
 * hierarchy, or a standalone single-level grid for plain Gauss-Seidel
 * (gs_parallel.cc:25-51).  The data lives on the GPU in libpgmg_b200.so;
 * this class keeps the reference's public fields and calls the C ABI.
 *
 * Differences from the reference, all for one process:
 *   - x0 / r0 (and x) are HOST MIRRORS of the device fields, natural order
 *     with no ghost layers (mg = m, ng = n, og = o, x0 = x).  pull() copies
 *     the device fields into them, push() copies them back; the methods of
 *     this class never touch the mirrors implicitly.
 *   - Problem-class stencils are copied at setup_matrices time; the
 *     reference instead aliases external_ptr() for the object's lifetime
 *     (region.hh:517).
 *   - Every error is reported through p_fatal_error, like the reference.
 */
#ifndef PGMG_REGION_HH
#define PGMG_REGION_HH

#include <cstring>
#include <vector>

#include "../pgmg_dev.h"
#include "buffer.hh"
#include "common.hh"
#include "geometry.hh"

namespace pgmg_dropin {

inline void check(pgmg_status st, pgmg_handle* h, const char* where) {
    if (st != PGMG_OK) {
        char msg[768];
        std::snprintf(msg, sizeof(msg), "pgmg %s failed (status %d): %s", where, (int)st,
                      h ? pgmg_dev_last_error(h) : "");
        p_fatal_error(msg, (int)st);
    }
}

/* Creates the device hierarchy.  Defaults: FP64, 8-colour smoother, LU on
 * the coarsest level.  PGMG_SMOOTHER=lex selects the reference's
 * lexicographic order (bit-for-bit the reference's sweeps) and
 * PGMG_COARSE=lu_exact|gs the reference-order LU solve or its 24-sweep
 * fallback. */
inline pgmg_handle* create(int m, int n, int o, bool xp, bool yp, bool zp) {
    pgmg_dims d;
    d.m = m; d.n = n; d.o = o;
    d.x_prd = xp; d.y_prd = yp; d.z_prd = zp;
    d.precision = PGMG_FP64;
    d.coarse = PGMG_COARSE_LU;
    d.smoother = PGMG_SMOOTH_MC8;
    d.device = -1;
    const char* sm = std::getenv("PGMG_SMOOTHER");
    if (sm && std::strcmp(sm, "lex") == 0) d.smoother = PGMG_SMOOTH_LEX;
    const char* co = std::getenv("PGMG_COARSE");
    if (co && std::strcmp(co, "lu_exact") == 0) d.coarse = PGMG_COARSE_LU_EXACT;
    if (co && std::strcmp(co, "gs") == 0) d.coarse = PGMG_COARSE_GS;
    pgmg_handle* h = 0;
    check(pgmg_dev_create(&d, &h), 0, "create");
    return h;
}

/* Reads the problem class (the duck-typed p_class concept of
 * problem_simple.hh:36-73) into natural-order boxes and 27-slot stencils. */
template <class p_class>
void read_boxes(p_class& pr, int m, int n, int o, std::vector<int>& S) {
    S.resize(6 * (size_t)m * n * o);
    int* sp = &S[0];
    for (int k = 0; k < o; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < m; i++) {
                *(sp++) = pr.range_xd(i, j, k);
                *(sp++) = pr.range_xu(i, j, k);
                *(sp++) = pr.range_yd(i, j, k);
                *(sp++) = pr.range_yu(i, j, k);
                *(sp++) = pr.range_zd(i, j, k);
                *(sp++) = pr.range_zu(i, j, k);
            }
}

template <class p_class>
void read_stencils(p_class& pr, int m, int n, int o, const std::vector<int>& S, std::vector<double>& c27) {
    c27.assign(27 * (size_t)m * n * o, 0.0);
    std::vector<double> tmp;
    size_t p = 0;
    for (int k = 0; k < o; k++)
        for (int j = 0; j < n; j++)
            for (int i = 0; i < m; i++, p++) {
                const int* s = &S[6 * p];
                int sz = (s[1] - s[0]) * (s[3] - s[2]) * (s[5] - s[4]);
                if (s[0] < -1 || s[1] > 2 || s[2] < -1 || s[3] > 2 || s[4] < -1 || s[5] > 2)
                    p_fatal_error("pgmg: stencil boxes must lie inside the 27-point neighbourhood", PGMG_SETUP_ERROR);
                const double* e;
                if (pr.internal(i, j, k)) {
                    /* region.hh:96-101: fill_entries writes mem_size entries. */
                    int ms = pr.mem_size(i, j, k);
                    if (ms != sz) p_fatal_error("pgmg: mem_size differs from the box size", PGMG_SETUP_ERROR);
                    tmp.resize(ms > 0 ? ms : 1);
                    double* en = &tmp[0];
                    pr.fill_entries(i, j, k, en);
                    e = &tmp[0];
                } else {
                    e = pr.external_ptr(i, j, k);
                }
                double* c = &c27[27 * p];
                for (int dk = s[4]; dk < s[5]; dk++)
                    for (int dj = s[2]; dj < s[3]; dj++)
                        for (int di = s[0]; di < s[1]; di++) c[(di + 1) + 3 * (dj + 1) + 9 * (dk + 1)] = *(e++);
            }
}

}  // namespace pgmg_dropin

class region {
   public:
    region* p;
    /* Sweep counter of region.cc:116 (C++17 inline variable). */
    inline static int gs_num = 0;
    int rank;
    const bool x_prd, y_prd, z_prd;
    bool gs_enable;
    const int m, n, o;
    const int ip, jp, kp, mp, np, op;
    double* x;
    double* x0;
    double* r0;
    int mg, ng, og, mng, indent;
    int ai, aj, ak, bi, bj, bk, sm, sn, so, smn, smno;
    MPI_Comm cart;

    /* Standalone top-level region from a problem class (region.hh:474-529). */
    template <class p_class>
    region(p_class& pr, geometry& gm, comm_buffer& com_)
        : p(0), rank(0), x_prd(gm.x_prd), y_prd(gm.y_prd), z_prd(gm.z_prd), gs_enable(true), m(gm.m), n(gm.n),
          o(gm.o), ip(0), jp(0), kp(0), mp(1), np(1), op(1), x(0), x0(0), r0(0), cart(gm.cart), h(0), level(0),
          owner(true), com(com_) {
        init_sizes();
        h = pgmg_dropin::create(m, n, o, x_prd, y_prd, z_prd);
        pgmg_dropin::read_boxes(pr, m, n, o, S);
    }
    /* Level `lev` of a hierarchy owned elsewhere (multigrid). */
    region(pgmg_handle* h_, int lev, region* parent, bool xp, bool yp, bool zp, comm_buffer& com_)
        : p(parent), rank(0), x_prd(xp), y_prd(yp), z_prd(zp), gs_enable(true), m(dims(h_, lev, 0)),
          n(dims(h_, lev, 1)), o(dims(h_, lev, 2)), ip(0), jp(0), kp(0), mp(1), np(1), op(1), x(0), x0(0), r0(0),
          cart(MPI_COMM_WORLD), h(h_), level(lev), owner(false), com(com_) {
        init_sizes();
    }
    ~region() {
        delete[] x;
        delete[] r0;
        if (owner && h) pgmg_dev_destroy(h);
    }

    template <class p_class>
    void setup_matrices(p_class& pr) {
        std::vector<double> c27;
        pgmg_dropin::read_stencils(pr, m, n, o, S, c27);
        pgmg_dropin::check(pgmg_dev_upload_level0(h, &c27[0], &S[0]), h, "upload_level0");
    }
    template <class p_class>
    void setup_fields(p_class& pr) {
        setup_x_field(pr);
        setup_r_field(pr);
    }
    template <class p_class>
    void setup_x_field(p_class& pr) {
        std::vector<double> v((size_t)smno);
        size_t q = 0;
        for (int k = 0; k < so; k++)
            for (int j = 0; j < sn; j++)
                for (int i = 0; i < sm; i++) v[q++] = pr.x_field(i, j, k);
        set(PGMG_FIELD_X, &v[0]);
    }
    template <class p_class>
    void setup_r_field(p_class& pr) {
        std::vector<double> v((size_t)smno);
        size_t q = 0;
        for (int k = 0; k < so; k++)
            for (int j = 0; j < sn; j++)
                for (int i = 0; i < sm; i++) v[q++] = pr.r_field(i, j, k);
        set(PGMG_FIELD_R, &v[0]);
    }
    template <class p_class>
    void overwrite_r_field(p_class& pr) {
        std::vector<double> v((size_t)smno);
        size_t q = 0;
        for (int k = 0; k < so; k++)
            for (int j = 0; j < sn; j++)
                for (int i = 0; i < sm; i++) v[q++] = pr.reset_r_field(i, j, k);
        set(PGMG_FIELD_R, &v[0]);
    }
    template <class p_class>
    void update_r_field(p_class& pr) {
        std::vector<double> v = get(PGMG_FIELD_R);
        size_t q = 0;
        for (int k = 0; k < so; k++)
            for (int j = 0; j < sn; j++)
                for (int i = 0; i < sm; i++) v[q++] += pr.update_r_field(i, j, k);
        set(PGMG_FIELD_R, &v[0]);
    }

    /* Host mirrors. */
    void pull() {
        alloc_mirrors();
        pgmg_dropin::check(pgmg_dev_get_field(h, level, PGMG_FIELD_X, x), h, "get_field");
        pgmg_dropin::check(pgmg_dev_get_field(h, level, PGMG_FIELD_R, r0), h, "get_field");
    }
    void push() {
        alloc_mirrors();
        set(PGMG_FIELD_X, x);
        set(PGMG_FIELD_R, r0);
    }

    void clear_r_field() {
        std::vector<double> z((size_t)smno, 0.0);
        set(PGMG_FIELD_R, &z[0]);
    }
    void clear_x_field() { pgmg_dropin::check(pgmg_dev_clear_x(h, level), h, "clear_x"); }
    void allclear_x_field() { clear_x_field(); }
    void copy_r_to_x() { pgmg_dropin::check(pgmg_dev_copy_r_to_x(h, level), h, "copy_r_to_x"); }
    void copy_x_to_r() {
        std::vector<double> v = get(PGMG_FIELD_X);
        set(PGMG_FIELD_R, &v[0]);
    }
    void communicate() {}
    void gauss_seidel(int mode = 0) {
        gs_num++;
        pgmg_dropin::check(pgmg_dev_gs(h, level, mode, -1), h, "gauss_seidel");
    }
    void solve_exact(bool smooth = 0) {
        if (smooth) {
            for (int l = 0; l < pgmg_gs_exact; l++) gauss_seidel();
        } else
            pgmg_dropin::check(pgmg_dev_coarse_solve(h), h, "solve_exact");
    }
    void restriction() { pgmg_dropin::check(pgmg_dev_restrict(h, level), h, "restriction"); }
    void interpolation() { pgmg_dropin::check(pgmg_dev_interp(h, level), h, "interpolation"); }
    /* Norms: sums of squares, no square root (region.cc:1475-1558). */
    double l2_error() { return norm(0); }
    double l2_error_all() { return norm(0); }
    double rhs_l2norm() { return norm(1); }
    double l0_error() {
        double e = 0;
        pgmg_dropin::check(pgmg_dev_l0_error(h, level, &e), h, "l0_error");
        return e;
    }
    double l0_error_all() { return l0_error(); }
    inline int total() { return m * n * o; }
    inline int min_size() { return sm < sn ? (sm < so ? sm : so) : (sn < so ? sn : so); }

    /* Output of a z-slice in the reference's float "binary matrix" layout
     * (region.cc:1638-1658): a header row [m, 0..m-1], then per row j the
     * value j followed by the m values. */
    void output_x(const char* filename, int k) { output(filename, k, get(PGMG_FIELD_X)); }
    void output_r(const char* filename, int k) { output(filename, k, get(PGMG_FIELD_R)); }
    void output_residual(const char* filename, int k) { output(filename, k, get(PGMG_FIELD_RES)); }
    void setup_test(int ca, bool xfield) {
        pgmg_dropin::check(pgmg_dev_setup_test(h, level, ca, xfield ? 1 : 0), h, "setup_test");
    }

    /* PCG helpers (region.cc:1848-1940), one process: the external arrays
     * have the x layout, which here is natural order. */
    void compute_residual(double* ext_r) {
        pgmg_dropin::check(pgmg_dev_get_field(h, level, PGMG_FIELD_RES, ext_r), h, "get_field");
    }
    void Ax(const double* in, double* out) { pgmg_dropin::check(pgmg_dev_apply(h, level, in, out), h, "apply"); }
    /* One process, no ghost padding: Ax wraps around periodic axes, which
     * is what unpadded_Ax does (region.cc:1876-1895). */
    void unpadded_Ax(const double* in, double* out) { Ax(in, out); }
    double source_soln_dot() {
        double s = 0;
        pgmg_dropin::check(pgmg_dev_source_soln_dot(h, level, &s), h, "source_soln_dot");
        return s;
    }
    void copy_rhs_to_soln() { copy_r_to_x(); }
    double soln_diff(double* ext_x) {
        double d = 0;
        pgmg_dropin::check(pgmg_dev_soln_diff(h, level, ext_x, &d), h, "soln_diff");
        return d;
    }
    void diagnostic_sums() {
        std::vector<double> res = get(PGMG_FIELD_RES), rr = get(PGMG_FIELD_R), xx = get(PGMG_FIELD_X);
        double su[6] = {0, 0, 0, 0, 0, 0};
        for (size_t q = 0; q < res.size(); q++) {
            su[0] += res[q]; su[1] += res[q] * res[q];
            su[2] += rr[q]; su[3] += rr[q] * rr[q];
            su[4] += xx[q]; su[5] += xx[q] * xx[q];
        }
        std::printf("Grid (%d,%d,%d): res (%g %g) r(%g %g) x(%g %g)\n", m, n, o, su[0], su[1], su[2], su[3], su[4],
                    su[5]);
    }
    pgmg_handle* handle() { return h; }
    int level_index() const { return level; }

   private:
    pgmg_handle* h;
    int level;
    bool owner;
    comm_buffer& com;
    std::vector<int> S;

    static int dims(pgmg_handle* hh, int lev, int a) {
        int d[3] = {0, 0, 0};
        pgmg_dropin::check(pgmg_dev_level_dims(hh, lev, d), hh, "level_dims");
        return d[a];
    }
    void init_sizes() {
        ai = aj = ak = 0;
        bi = sm = m; bj = sn = n; bk = so = o;
        smn = sm * sn; smno = smn * so;
        mg = m; ng = n; og = o; mng = mg * ng; indent = 0;
    }
    void alloc_mirrors() {
        if (!x) {
            x = new double[(size_t)smno];
            x0 = x;
            r0 = new double[(size_t)smno];
        }
    }
    std::vector<double> get(int field) {
        std::vector<double> v((size_t)smno);
        pgmg_dropin::check(pgmg_dev_get_field(h, level, field, &v[0]), h, "get_field");
        return v;
    }
    void set(int field, const double* v) { pgmg_dropin::check(pgmg_dev_set_field(h, level, field, v), h, "set_field"); }
    double norm(int which) {
        double a = 0, b = 0;
        pgmg_dropin::check(pgmg_dev_norms(h, level, &a, &b), h, "norms");
        return which ? b : a;
    }
    void output(const char* filename, int k, const std::vector<double>& v) {
        if (k < 0 || k >= o) p_fatal_error("Output slice out of range", 1);
        FILE* f = p_safe_fopen(filename, "wb");
        std::vector<float> buf((size_t)m + 1);
        buf[0] = (float)m;
        for (int i = 0; i < m; i++) buf[i + 1] = (float)i;
        if (std::fwrite(&buf[0], sizeof(float), m + 1, f) != (size_t)m + 1) p_fatal_error("File output error", 1);
        for (int j = 0; j < n; j++) {
            buf[0] = (float)j;
            for (int i = 0; i < m; i++) buf[i + 1] = (float)v[i + (size_t)m * (j + (size_t)n * k)];
            if (std::fwrite(&buf[0], sizeof(float), m + 1, f) != (size_t)m + 1) p_fatal_error("File output error", 1);
        }
        std::fclose(f);
    }
    region(const region&);
    region& operator=(const region&);
};

#endif
