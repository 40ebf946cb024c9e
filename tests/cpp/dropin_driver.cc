// Drop-in check: a driver written against the reference's C++ interface
// (as guide_test.cc, mg_parallel.cc, gs_parallel.cc and mg_test.cc use it),
// compiled against include/pgmg/ and run on the GPU.  The problem is read
// from a binary file: int m,n,o; then per point 6 int box bounds and 27
// doubles (slot (di+1)+3(dj+1)+9(dk+1)), then m*n*o doubles of source.
#include <cstdio>
#include <vector>

#include "mpi.h"
#include "multigrid.hh"

// A problem class of the reference's concept whose points are all
// "internal" (fill_entries, region.hh:96-101).
struct file_problem {
    bool x_prd, y_prd, z_prd;
    int m, n, o;
    std::vector<int> S;
    std::vector<double> c, r;
    explicit file_problem(const char* fn) : x_prd(false), y_prd(false), z_prd(false) {
        FILE* f = std::fopen(fn, "rb");
        if (!f) p_fatal_error("cannot open problem file", 1);
        int d[3];
        if (std::fread(d, sizeof(int), 3, f) != 3) p_fatal_error("bad problem file", 1);
        m = d[0]; n = d[1]; o = d[2];
        size_t N = (size_t)m * n * o;
        S.resize(6 * N); c.resize(27 * N); r.resize(N);
        if (std::fread(&S[0], sizeof(int), 6 * N, f) != 6 * N || std::fread(&c[0], sizeof(double), 27 * N, f) != 27 * N ||
            std::fread(&r[0], sizeof(double), N, f) != N)
            p_fatal_error("bad problem file", 1);
        std::fclose(f);
    }
    size_t id(int i, int j, int k) const { return i + (size_t)m * (j + (size_t)n * k); }
    int range_xd(int i, int j, int k) { return S[6 * id(i, j, k)]; }
    int range_xu(int i, int j, int k) { return S[6 * id(i, j, k) + 1]; }
    int range_yd(int i, int j, int k) { return S[6 * id(i, j, k) + 2]; }
    int range_yu(int i, int j, int k) { return S[6 * id(i, j, k) + 3]; }
    int range_zd(int i, int j, int k) { return S[6 * id(i, j, k) + 4]; }
    int range_zu(int i, int j, int k) { return S[6 * id(i, j, k) + 5]; }
    bool internal(int, int, int) { return true; }
    int mem_size(int i, int j, int k) {
        const int* s = &S[6 * id(i, j, k)];
        return (s[1] - s[0]) * (s[3] - s[2]) * (s[5] - s[4]);
    }
    void fill_entries(int i, int j, int k, double*& en) {
        const int* s = &S[6 * id(i, j, k)];
        const double* cc = &c[27 * id(i, j, k)];
        for (int dk = s[4]; dk < s[5]; dk++)
            for (int dj = s[2]; dj < s[3]; dj++)
                for (int di = s[0]; di < s[1]; di++) *(en++) = cc[(di + 1) + 3 * (dj + 1) + 9 * (dk + 1)];
    }
    double* external_ptr(int, int, int) { return 0; }
    double x_field(int, int, int) { return 0; }
    double r_field(int i, int j, int k) { return r[id(i, j, k)]; }
};

int main(int argc, char* argv[]) {
    MPI_Init(&argc, &argv);
    if (argc < 3) p_fatal_error("usage: dropin_driver problem.bin outdir", 1);
    file_problem pr(argv[1]);
    comm_buffer com;
    geometry gm(pr.m, pr.n, pr.o, false, false, false);
    multigrid mg(pr, gm, com);
    mg.setup_matrices(pr);
    mg.setup_fields(pr);
    std::printf("levels %d\n", mg.nlevels);
    for (int l = 0; l < mg.nlevels; l++) std::printf("dims %d %d %d %d\n", l, mg.reg[l]->m, mg.reg[l]->n, mg.reg[l]->o);
    for (int it = 0; it < 3; it++) {
        mg.v_cycle();
        std::printf("vcycle %d %.17g\n", it, mg.l2_error_all());
    }
    std::printf("rhs %.17g\n", mg.rhs_l2norm());
    char fn[512];
    std::snprintf(fn, sizeof(fn), "%s/x.slice", argv[2]);
    mg.output_x(fn, pr.o / 2);
    // Ax of the current solution equals r - residual.
    size_t N = (size_t)pr.m * pr.n * pr.o;
    std::vector<double> xin(N), ax(N), res(N);
    mg.reg[0]->pull();
    for (size_t q = 0; q < N; q++) xin[q] = mg.reg[0]->x0[q];
    mg.Ax(&xin[0], &ax[0]);
    mg.compute_residual(&res[0]);
    double worst = 0;
    for (size_t q = 0; q < N; q++) {
        double d = std::fabs(ax[q] + res[q] - mg.reg[0]->r0[q]);
        worst = d > worst ? d : worst;
    }
    std::printf("ax_check %.3g\n", worst);
    // solve_v_cycles with the guide (guide_test.cc:24-36), twice.
    mg.guide.set_tol(8.0 / 3.0 / (pr.m - 1));
    for (int rep = 0; rep < 2; rep++) {
        mg.setup_fields(pr);
        double resid;
        int st = mg.solve_v_cycles(resid);
        std::printf("solve %d %d %.17g %d\n", rep, st, resid, mg.guide.pred_iters());
    }
    // Standalone region, plain sweeps (gs_parallel.cc:25-40).
    region rg(pr, gm, com);
    rg.setup_matrices(pr);
    rg.setup_fields(pr);
    std::printf("gs 0 %.17g\n", rg.l2_error());
    for (int s = 1; s <= 3; s++) {
        rg.gauss_seidel();
        std::printf("gs %d %.17g\n", s, rg.l2_error());
    }
    mg.free();
    gm.free();
    MPI_Finalize();
    return 0;
}
