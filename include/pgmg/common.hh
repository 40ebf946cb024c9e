/* Drop-in common definitions (reference common.hh:12-65): tuning constants,
 * error codes and the fatal-error helpers, for one process. */
#ifndef PGMG_COMMON_HH
#define PGMG_COMMON_HH

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>

#include "mpi.h"

const int mg_max_levels = 16;
const MPI_Comm world = MPI_COMM_WORLD;

enum { PGMG_FILE_ERROR, PGMG_MEMORY_ERROR, PGMG_INTERNAL_ERROR, PGMG_MULTIGRID_ERROR, PGMG_MATH_ERROR, PGMG_SETUP_ERROR };

#define PGMG_VERBOSE 1
const double pgmg_exact_tol = std::numeric_limits<double>::epsilon() * 1e4;
const int pgmg_gs_exact = 24;
const int pgmg_max_exact = 2048;

inline FILE* safe_fopen(const char* filename, const char* mode) {
    FILE* f = std::fopen(filename, mode);
    if (!f) {
        std::fprintf(stderr, "Error opening file \"%s\"", filename);
        std::exit(1);
    }
    return f;
}
inline FILE* p_safe_fopen(const char* filename, const char* mode) {
    FILE* f = std::fopen(filename, mode);
    if (!f) {
        std::fprintf(stderr, "Unable to open file '%s'\n", filename);
        MPI_Abort(world, PGMG_FILE_ERROR);
    }
    return f;
}
inline void fatal_error(const char* p, int code) {
    std::fprintf(stderr, "Error: %s\n", p);
    std::exit(code);
}
inline void p_fatal_error(const char* p, int status) {
    std::fprintf(stderr, "%s\n", p);
    MPI_Abort(world, status);
}
inline void p_die() { p_fatal_error("Died", PGMG_INTERNAL_ERROR); }

#endif
