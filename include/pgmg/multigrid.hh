/* Drop-in multigrid (reference multigrid.hh:20-321) on one GPU.
 *
 * Same construction and calls as the reference:
 *     geometry gm(m, n, o, false, false, false);
 *     my_problem pr(gm);
 *     comm_buffer com;
 *     multigrid mg(pr, gm, com);     // hierarchy planned, device arena allocated
 *     mg.setup_matrices(pr);         // level-0 stencils uploaded, RAT + LU on the GPU
 *     mg.setup_fields(pr);
 *     mg.guide.set_tol(p_scale);
 *     int st = mg.solve_v_cycles(res);
 * The public tuning fields v_down / v_up / v_bottom and the mg_guide struct
 * behave as in the reference.  reg[l] are drop-in regions (see region.hh for
 * the host-mirror convention of x0 / r0).  Build with -std=c++17 and link
 * libpgmg_b200.so.
 */
#ifndef PGMG_MULTI_HH
#define PGMG_MULTI_HH

#include <limits>

#include "buffer.hh"
#include "common.hh"
#include "geometry.hh"
#include "region.hh"

class multigrid {
   public:
    /* multigrid.hh:34-118, unchanged semantics. */
    struct mg_guide {
        static const int DEF_PERIOD = 16;
        static const int INIT_VAR = 1000000;
        static const int DEF_ALPHA = 3;
        static const int MAX_ITERS = 100;
        static const int FUDGE_FACTOR = 10000;
        static const int INSURANCE = 2;
        int period, iter;
        bool use_avg;
        double iter_avg, iter_var, alpha, tol;
        bool tol_set_manually;
        mg_guide() : use_avg(false), tol_set_manually(false) {
            set_period(DEF_PERIOD);
            alpha = (1. * DEF_ALPHA) / period;
        }
        inline void set_tol(double p_scale) {
            double eps = std::numeric_limits<double>::epsilon();
            tol = p_scale * p_scale * eps * eps * FUDGE_FACTOR;
            tol_set_manually = true;
        }
        inline void average_on() { use_avg = true; }
        inline void average_on(double alpha_) { use_avg = true; alpha = alpha_; }
        inline void average_off() { use_avg = false; }
        inline void set_period(int period_) {
            period = period_;
            iter_avg = iter = period;
            iter_var = INIT_VAR;
        }
        /* multigrid.cc:268-293 */
        void update(int extras) {
            int diter = -1 + period * extras;
            if (use_avg) {
                double di = iter - iter_avg;
                int zscore = static_cast<int>(di / std::sqrt(iter_var));
                if (zscore > 0) diter -= zscore;
                iter_avg = (1 - alpha) * iter_avg + alpha * iter;
                iter_var = (1 - alpha) * (iter_var + alpha * di * di);
            }
            iter += diter;
            if (iter < period) iter = 2 * period - 1;
        }
        inline int pred_iters() { return iter / period; }
    };

    int v_down, v_bottom, v_up, rank, nlevels, mlevels;
    mg_guide guide;
    geometry* geom;
    region** reg;
    geometry** geo;

    template <class p_class>
    multigrid(p_class& pr, geometry& gm, comm_buffer& com_)
        : v_down(2), v_bottom(20), v_up(2), rank(0), nlevels(0), mlevels(0), geom(&gm), reg(0), geo(0), com(com_),
          h(0), pushed_down(-1), pushed_up(-1), pushed_bottom(-1) {
        h = pgmg_dropin::create(gm.m, gm.n, gm.o, gm.x_prd, gm.y_prd, gm.z_prd);
        pgmg_dropin::check(pgmg_dev_num_levels(h, &nlevels), h, "num_levels");
        mlevels = nlevels;
        reg = new region*[mg_max_levels];
        geo = new geometry*[mg_max_levels];
        for (int l = 0; l < mg_max_levels; l++) {
            reg[l] = 0;
            geo[l] = 0;
        }
        for (int l = 0; l < nlevels; l++)
            reg[l] = new region(h, l, l ? reg[l - 1] : 0, gm.x_prd, gm.y_prd, gm.z_prd, com);
        pgmg_dropin::read_boxes(pr, gm.m, gm.n, gm.o, S);
    }
    ~multigrid() {
        for (int l = nlevels - 1; l >= 0; l--) delete reg[l];
        delete[] reg;
        delete[] geo;
        if (h) pgmg_dev_destroy(h);
    }

    /* multigrid.hh:302-305: level-0 stencils, then every Galerkin operator
     * and the coarsest LU, on the GPU. */
    template <class p_class>
    void setup_matrices(p_class& pr) {
        std::vector<double> c27;
        pgmg_dropin::read_stencils(pr, geom->m, geom->n, geom->o, S, c27);
        pgmg_dropin::check(pgmg_dev_upload_level0(h, &c27[0], &S[0]), h, "upload_level0");
        compute_rats();
    }
    template <class p_class>
    void setup_fields(p_class& pr) { reg[0]->setup_fields(pr); }
    template <class p_class>
    void setup_r_field(p_class& pr) { reg[0]->setup_r_field(pr); }
    template <class p_class>
    void update_r_field(p_class& pr) { reg[0]->update_r_field(pr); }
    template <class p_class>
    void overwrite_r_field(p_class& pr) { reg[0]->overwrite_r_field(pr); }
    inline void allclear_x_field() { reg[0]->allclear_x_field(); }
    void compute_rats() { pgmg_dropin::check(pgmg_dev_build_rat(h), h, "build_rat"); }
    void setup_hierarchy(geometry&) {}

    void v_cycle(int mode = 0) {
        push_schedule();
        pgmg_dropin::check(pgmg_dev_vcycle(h, mode, -1), h, "v_cycle");
    }
    void fmg_cycle() {
        push_schedule();
        pgmg_dropin::check(pgmg_dev_fmg_cycle(h, -1), h, "fmg_cycle");
    }
    double l2_error(int level = 0) { return level < nlevels ? reg[level]->l2_error() : 0; }
    double l2_error_all(int level = 0) { return level < nlevels ? reg[level]->l2_error_all() : 0; }
    double l0_error(int level = 0) { return level < nlevels ? reg[level]->l0_error() : 0; }
    double l0_error_all(int level = 0) { return level < nlevels ? reg[level]->l0_error_all() : 0; }
    double rhs_l2norm(int level = 0) { return level < nlevels ? reg[level]->rhs_l2norm() : 0; }
    void gauss_seidel(int mode = 0, int level = 0) {
        if (level < nlevels && reg[level]->gs_enable) reg[level]->gauss_seidel(mode);
    }

    /* multigrid.hh:182-219, the same loop over device V-cycles. */
    int solve_v_cycles(double& res) {
        if (!guide.tol_set_manually)
            p_fatal_error("multigrid::solve_v_cycles cannot be used before the class mg_guide instance uses"
                          " the function multigrid::mg_pred::set_tol to set the target tolerance to be reached", 1);
        double tol = guide.tol * geom->m;
        tol *= geom->n;
        tol *= geom->o;
        for (int i = 0; i < guide.pred_iters(); i++) v_cycle();
        int extra_rounds = 0, n = 0;
        while ((res = l2_error_all()) > tol && n < guide.MAX_ITERS) {
            if (std::isnan(res)) return 2;
            extra_rounds++;
            for (int i = 0; i < extra_rounds; i++, n++) v_cycle();
        }
        if (n > guide.MAX_ITERS) return 1;
        for (int i = 0; i < guide.INSURANCE; i++) v_cycle();
        guide.update(extra_rounds * (extra_rounds + 1) / 2);
        return 0;
    }
    int solve_v_cycles() {
        double res;
        return solve_v_cycles(res);
    }
    /* Relative-residual solve on the device (this library's addition):
     * V-cycles until sqrt(sum r^2 / sum b^2) < tol.  Returns the cycles run. */
    int solve(double tol, int max_cycles = 100, double* relres = 0) {
        push_schedule();
        int cyc = 0;
        double rr = 0;
        pgmg_dropin::check(pgmg_dev_solve_relres(h, tol, max_cycles, 0, &cyc, &rr), h, "solve_relres");
        if (relres) *relres = rr;
        return cyc;
    }

    inline void compute_residual(double* ext_r) { reg[0]->compute_residual(ext_r); }
    void Ax(const double* in, double* out) { reg[0]->Ax(in, out); }
    void unpadded_Ax(const double* in, double* out, const int lev = 0) {
        if (lev >= nlevels) p_fatal_error("Unpadded_Ax only available within multigrid hierarchy.", 1);
        reg[lev]->unpadded_Ax(in, out);
    }
    void copy_rhs_to_soln() { reg[0]->copy_rhs_to_soln(); }
    double source_soln_dot() { return reg[0]->source_soln_dot(); }
    double soln_diff(double* ext_x) { return reg[0]->soln_diff(ext_x); }

    void interpolation(int level) {
        if (level < nlevels) reg[level]->interpolation();
    }
    void restriction(int level) {
        if (level < nlevels) reg[level]->restriction();
    }
    void communicate(int = 0) {}
    void output_x(const char* filename, int k, int level = 0) {
        if (level < nlevels) reg[level]->output_x(filename, k);
    }
    void output_r(const char* filename, int k, int level = 0) {
        if (level < nlevels) reg[level]->output_r(filename, k);
    }
    void output_residual(const char* filename, int k, int level = 0) {
        if (level < nlevels) reg[level]->output_residual(filename, k);
    }
    inline void solve_exact(int level = 0, bool smooth = 0) {
        if (level < nlevels) {
            if (smooth || level != nlevels - 1) {
                for (int l = 0; l < pgmg_gs_exact; l++) reg[level]->gauss_seidel();
            } else
                reg[level]->solve_exact(false);
        }
    }
    inline void free() {}
    inline void setup_test(int ca, bool xfield, int level = 0) {
        if (level < nlevels) reg[level]->setup_test(ca, xfield);
    }
    inline void diagnostic_sums(int level = 0) {
        if (level < nlevels) reg[level]->diagnostic_sums();
    }
    pgmg_handle* handle() { return h; }

   protected:
    comm_buffer& com;

   private:
    pgmg_handle* h;
    std::vector<int> S;
    int pushed_down, pushed_up, pushed_bottom;
    /* The public sweep counts are read at every cycle, as the reference reads
     * its fields in v_cycle (multigrid.cc:92,102). */
    void push_schedule() {
        if (v_down != pushed_down) {
            pgmg_dropin::check(pgmg_dev_set_option(h, PGMG_OPT_V_DOWN, v_down), h, "set_option");
            pushed_down = v_down;
        }
        if (v_up != pushed_up) {
            pgmg_dropin::check(pgmg_dev_set_option(h, PGMG_OPT_V_UP, v_up), h, "set_option");
            pushed_up = v_up;
        }
        if (v_bottom != pushed_bottom) {
            pgmg_dropin::check(pgmg_dev_set_option(h, PGMG_OPT_V_BOTTOM, v_bottom), h, "set_option");
            pushed_bottom = v_bottom;
        }
    }
    multigrid(const multigrid&);
    multigrid& operator=(const multigrid&);
};

#endif
