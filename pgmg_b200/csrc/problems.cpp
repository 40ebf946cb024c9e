// Host-side problem generators: the synthetic inputs of the benchmark
// configurations, written as the reference's problem-class concept would
// supply them (per-point stencil box + coefficients, sources, Dirichlet fix
// rows; problem_simple.hh:36-73).  The reference ships no variable-coefficient
// class (fill_entries is fatal in problem_simple.cc:10-12), so these are this
// library's own classes; the oracle consumes the same arrays.
//
//  * kappa field: cell-centred g ~ N(0,1) i.i.d. per cell from a counter-based
//    generator (SplitMix64 of seed ^ counter, Box-Muller), convolved with a
//    separable Gaussian of width 8 cells truncated at 4 widths with
//    half-sample-symmetric (reflective) edges, normalised to zero mean and
//    unit variance, kappa = exp(sigma*g).
//  * Q1 trilinear FEM stencil of -div(kappa grad u): each interior node sums
//    h*kappa_e*K^ over its 8 cells, K^ = 1/3 on the diagonal, 0 for nodes one
//    coordinate apart, -1/12 for two or three coordinates apart (constant
//    kappa gives centre 8/3 h, face 0, edge -h/6, corner -h/12).  h =
//    1/(max(m,n,o)-1).
//  * Dirichlet boundary nodes are one-entry "fix" rows (box [0,1)^3), as in
//    problem_simple.hh:36-41,65-67, with a positive value 8/3*h*mean(kappa of
//    the cells touching the node), and right-hand side 0.
//  * RHS: interior nodes i.i.d. uniform[-1,1] from SplitMix64(seed ^ index).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/pgmg_dev.h"

namespace {

inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Uniform in (0,1]: 53 random bits, offset by one ulp so log() is finite.
inline double unit_open0(uint64_t bits) {
    return ((bits >> 11) + 1) * (1.0 / 9007199254740992.0);
}

// Half-sample-symmetric reflection of index t into [0,len).
inline long reflect(long t, long len) {
    if (len == 1) return 0;
    long period = 2 * len;
    t %= period;
    if (t < 0) t += period;
    return t < len ? t : period - 1 - t;
}

void smooth_axis(std::vector<double>& a, long nx, long ny, long nz, int axis,
                 const std::vector<double>& w, int rad) {
    long len = axis == 0 ? nx : (axis == 1 ? ny : nz);
    long stride = axis == 0 ? 1 : (axis == 1 ? nx : nx * ny);
    long lines = nx * ny * nz / len;
    std::vector<double> out(a.size());
#pragma omp parallel for schedule(static)
    for (long l = 0; l < lines; l++) {
        long base;
        if (axis == 0) base = l * nx;
        else if (axis == 1) base = (l / nx) * nx * ny + (l % nx);
        else base = l;
        for (long t = 0; t < len; t++) {
            double s = 0;
            for (int d = -rad; d <= rad; d++) s += w[d + rad] * a[base + reflect(t + d, len) * stride];
            out[base + t * stride] = s;
        }
    }
    a.swap(out);
}

}  // namespace

extern "C" {

int pgmg_problem_kappa(int m, int n, int o, double sigma, uint64_t seed, double width, double* kappa) {
    if (m < 2 || n < 2 || o < 2 || !kappa) return PGMG_ERR_ARG;
    int st = pgmg_problem_gauss(m, n, o, seed, width, kappa);
    if (st) return st;
    long nc = (long)(m - 1) * (n - 1) * (o - 1);
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nc; c++) kappa[c] = std::exp(sigma * kappa[c]);
    return PGMG_OK;
}

int pgmg_problem_gauss(int m, int n, int o, uint64_t seed, double width, double* out) {
    if (m < 2 || n < 2 || o < 2 || !out) return PGMG_ERR_ARG;
    long nx = m - 1, ny = n - 1, nz = o - 1, nc = nx * ny * nz;
    std::vector<double> g(nc);
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nc; c++) {
        uint64_t key = seed * 0x100000001B3ull;
        double u1 = unit_open0(splitmix64(key ^ (2 * (uint64_t)c)));
        double u2 = unit_open0(splitmix64(key ^ (2 * (uint64_t)c + 1)));
        g[c] = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
    if (width > 0) {
        int rad = (int)std::ceil(4 * width);
        std::vector<double> w(2 * rad + 1);
        double ws = 0;
        for (int d = -rad; d <= rad; d++) ws += (w[d + rad] = std::exp(-0.5 * d * d / (width * width)));
        for (double& v : w) v /= ws;
        smooth_axis(g, nx, ny, nz, 0, w, rad);
        smooth_axis(g, nx, ny, nz, 1, w, rad);
        smooth_axis(g, nx, ny, nz, 2, w, rad);
    }
    // Deterministic normalisation: per-plane partial sums, then a serial sum.
    std::vector<double> ps(nz), pq(nz);
#pragma omp parallel for schedule(static)
    for (long k = 0; k < nz; k++) {
        double s = 0;
        for (long c = k * nx * ny; c < (k + 1) * nx * ny; c++) s += g[c];
        ps[k] = s;
    }
    double mean = 0;
    for (long k = 0; k < nz; k++) mean += ps[k];
    mean /= (double)nc;
#pragma omp parallel for schedule(static)
    for (long k = 0; k < nz; k++) {
        double q = 0;
        for (long c = k * nx * ny; c < (k + 1) * nx * ny; c++) q += (g[c] - mean) * (g[c] - mean);
        pq[k] = q;
    }
    double var = 0;
    for (long k = 0; k < nz; k++) var += pq[k];
    var /= (double)nc;
    double inv_sd = var > 0 ? 1.0 / std::sqrt(var) : 0.0;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nc; c++) out[c] = (g[c] - mean) * inv_sd;
    return PGMG_OK;
}

int pgmg_problem_q1(int m, int n, int o, const double* kappa, double* coef27, int* S6) {
    if (m < 2 || n < 2 || o < 2 || !coef27) return PGMG_ERR_ARG;
    const long nx = m - 1, ny = n - 1;
    const double h = 1.0 / (double)((m > n ? (m > o ? m : o) : (n > o ? n : o)) - 1);
    // K^ by number of differing coordinates.
    const double khat[4] = {1.0 / 3.0, 0.0, -1.0 / 12.0, -1.0 / 12.0};
    auto kap = [&](long ci, long cj, long ck) -> double {
        return kappa ? kappa[ci + nx * (cj + ny * ck)] : 1.0;
    };
#pragma omp parallel for schedule(static)
    for (long k = 0; k < o; k++)
        for (long j = 0; j < n; j++)
            for (long i = 0; i < m; i++) {
                long p = i + (long)m * (j + (long)n * k);
                double* c = coef27 + 27 * p;
                for (int q = 0; q < 27; q++) c[q] = 0;
                bool interior = i > 0 && i < m - 1 && j > 0 && j < n - 1 && k > 0 && k < o - 1;
                if (interior) {
                    // The 8 cells around the node: cell (i+ca, j+cb, k+ce) with
                    // ca,cb,ce in {-1,0}; the node is that cell's local corner
                    // (-ca,-cb,-ce), the cell's other corner (aa,bb,ee) is the
                    // node at offset (aa+ca, bb+cb, ee+ce).
                    for (int ce = -1; ce <= 0; ce++)
                        for (int cb = -1; cb <= 0; cb++)
                            for (int ca = -1; ca <= 0; ca++) {
                                double ke = h * kap(i + ca, j + cb, k + ce);
                                for (int ee = 0; ee < 2; ee++)
                                    for (int bb = 0; bb < 2; bb++)
                                        for (int aa = 0; aa < 2; aa++) {
                                            int diff = (aa != -ca) + (bb != -cb) + (ee != -ce);
                                            int q = (aa + ca + 1) + 3 * (bb + cb + 1) + 9 * (ee + ce + 1);
                                            c[q] += ke * khat[diff];
                                        }
                            }
                } else {
                    double s = 0;
                    int cnt = 0;
                    for (int e = -1; e <= 0; e++)
                        for (int b = -1; b <= 0; b++)
                            for (int a = -1; a <= 0; a++) {
                                long ci = i + a, cj = j + b, ck = k + e;
                                if (ci < 0 || cj < 0 || ck < 0 || ci >= nx || cj >= ny || ck >= o - 1) continue;
                                s += kap(ci, cj, ck);
                                cnt++;
                            }
                    c[13] = 8.0 / 3.0 * h * (s / cnt);
                }
                if (S6) {
                    int* s = S6 + 6 * p;
                    s[0] = s[2] = s[4] = interior ? -1 : 0;
                    s[1] = s[3] = s[5] = interior ? 2 : 1;
                }
            }
    return PGMG_OK;
}

int pgmg_problem_rhs(int m, int n, int o, uint64_t seed, double* r) {
    if (m < 1 || n < 1 || o < 1 || !r) return PGMG_ERR_ARG;
    uint64_t key = (seed + 0x5851F42D4C957F2Dull) * 0x2545F4914F6CDD1Dull;
#pragma omp parallel for schedule(static)
    for (long k = 0; k < o; k++)
        for (long j = 0; j < n; j++)
            for (long i = 0; i < m; i++) {
                long p = i + (long)m * (j + (long)n * k);
                bool interior = i > 0 && i < m - 1 && j > 0 && j < n - 1 && k > 0 && k < o - 1;
                r[p] = interior ? 2.0 * (unit_open0(splitmix64(key ^ (uint64_t)p)) - 0.5) : 0.0;
            }
    return PGMG_OK;
}

}  // extern "C"
