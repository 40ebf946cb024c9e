/* Single-process MPI compatibility for programs written against the PGMG
 * reference (which includes "mpi.h" from every file, common.hh:8).  This
 * library runs one process per GPU and has no MPI on its path; driver
 * programs keep their MPI_Init / MPI_Wtime / MPI_Barrier / MPI_Finalize calls
 * and get one rank.  Only what those drivers and the drop-in headers use is
 * provided. */
#ifndef PGMG_DROPIN_MPI_H
#define PGMG_DROPIN_MPI_H

#include <cstdio>
#include <cstdlib>
#include <time.h>

typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_SUCCESS 0

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Abort(MPI_Comm, int code) {
    std::fprintf(stderr, "MPI_Abort(%d)\n", code);
    std::exit(code == 0 ? 1 : code);
    return code;
}
inline double MPI_Wtime() {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

#endif
