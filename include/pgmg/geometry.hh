/* Drop-in geometry (reference geometry.hh:8-77) for one process: the whole
 * grid belongs to rank 0 (procs = mp = np = op = 1). */
#ifndef PGMG_GEOMETRY_HH
#define PGMG_GEOMETRY_HH

#include "common.hh"

class geometry {
   public:
    const int m, n, o;
    const bool x_prd, y_prd, z_prd;
    int rank, procs, mp, np, op, ip, jp, kp;
    int ai, aj, ak, bi, bj, bk, sm, sn, so, smn, smno;
    MPI_Comm cart;
    int* ranks;
    /* geometry.cc:12-26 */
    geometry(int m_, int n_, int o_, bool x_prd_, bool y_prd_, bool z_prd_)
        : m(m_), n(n_), o(o_), x_prd(x_prd_), y_prd(y_prd_), z_prd(z_prd_), ranks(0) {
        init();
    }
    /* The "+1" copy (geometry.cc:76-95): one more point on every
     * non-periodic axis. */
    geometry(const geometry& gm)
        : m(gm.x_prd ? gm.m : gm.m + 1), n(gm.y_prd ? gm.n : gm.n + 1), o(gm.z_prd ? gm.o : gm.o + 1),
          x_prd(gm.x_prd), y_prd(gm.y_prd), z_prd(gm.z_prd), ranks(0) {
        init();
    }
    void free() {}
    /* geometry.cc:164-172 on a 1x1x1 process grid. */
    void set_up_neighbors(int* neigh) {
        for (int k = -1; k <= 1; k++)
            for (int j = -1; j <= 1; j++)
                for (int i = -1; i <= 1; i++, neigh++)
                    *neigh = ((z_prd || k == 0) && (y_prd || j == 0) && (x_prd || i == 0)) ? 0 : -1;
    }

   private:
    void init() {
        rank = 0; procs = 1; mp = np = op = 1; ip = jp = kp = 0;
        ai = aj = ak = 0; bi = m; bj = n; bk = o;
        sm = m; sn = n; so = o; smn = sm * sn; smno = smn * so;
        cart = MPI_COMM_WORLD;
    }
};

#endif
