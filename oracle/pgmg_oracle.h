/* CPU restatement of the PGMG reference multigrid hot path (oracle).
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py as the checker.  The product never links it.
 *
 * Scope: one process, non-periodic axes, stencil boxes inside [-1,2)^3 (the
 * 27-point neighbourhood), FP64.  Storage: 27 coefficient slots per point
 * (slot (di+1)+3(dj+1)+9(dk+1), zero outside the point's box), natural order
 * with i fastest; per-point boxes kept as 6 ints [xd,xu,yd,yu,zd,zu].
 * Parity status: pinned against the reference compiled from its own sources
 * (oracle/_ref/libpgmg_ref.so) by tests/test_oracle_pin.py.
 */
#ifndef PGMG_ORACLE_H
#define PGMG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc orc;

/* coarse: 1 = factorise the bottom level with LU after the Galerkin build
 * (falling back to 24 Gauss-Seidel sweeps if the conditioning check fails),
 * 0 = always 24 Gauss-Seidel sweeps (the reference's fallback path). */
orc* orc_create(int m,int n,int o,const int *S6,const double *c27,const double *r,
		const double *x,int coarse);
void orc_destroy(orc *h);
int orc_nlevels(orc *h);
void orc_level_dims(orc *h,int l,int *mno);
int orc_lu_enabled(orc *h);
void orc_get_x(orc *h,int l,double *out);
void orc_set_x(orc *h,int l,const double *in);
void orc_get_r(orc *h,int l,double *out);
void orc_set_r(orc *h,int l,const double *in);
void orc_get_S(orc *h,int l,int *out);
void orc_get_A27(orc *h,int l,double *out);
void orc_gauss_seidel(orc *h,int mode,int l);
void orc_gauss_seidel_mc8(orc *h,int mode,int l);
/* Smoother of orc_v_cycle and of the coarse fallback sweeps: 0 = the
 * reference's lexicographic Gauss-Seidel (default), 1 = 8-colour. */
void orc_set_smoother(orc *h,int mc8);
/* Slab budget of the 8-colour sweep in bytes of FP64 solution vector
 * (default 0 = one slab, the library's default). */
void orc_set_slab_budget(orc *h,long long bytes);
void orc_restriction(orc *h,int l);
void orc_interpolation(orc *h,int l);
void orc_solve_exact(orc *h,int l);
void orc_v_cycle(orc *h,int mode);
double orc_l2_error_all(orc *h,int l);
double orc_rhs_l2norm(orc *h,int l);
int orc_solve_v_cycles(orc *h,double p_scale,double *res,long *sweeps);
void orc_setup_test(orc *h,int ca,int xfield,int l);
void orc_clear_x(orc *h,int l);
int orc_guide_pred_iters(orc *h);
/* Seeded benchmark inputs (oracle/inputs.c): the same arrays as the
 * library's host generators, bit for bit, so that the reference arm of the
 * benchmark never loads the product library.  Return 0 on success. */
int orc_input_gauss(int m,int n,int o,uint64_t seed,double width,double *out);
int orc_input_kappa(int m,int n,int o,double sigma,uint64_t seed,double width,double *kappa);
int orc_input_q1(int m,int n,int o,const double *kappa,double *c27,int *S6);
int orc_input_rhs(int m,int n,int o,uint64_t seed,double *r);
/* Plain dense LU pieces, exposed for the coarse-solver tests. */
int orc_dgetrf(int n,double *a,int *ipiv);
void orc_dgetrs(int n,const double *a,const int *ipiv,double *b);

#ifdef __cplusplus
}
#endif

#endif
