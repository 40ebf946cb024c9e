/* C-ABI driver around the UNMODIFIED PGMG reference multigrid, compiled into
 * oracle/_ref/libpgmg_ref.so by oracle/Makefile from the reference's own
 * sources (buffer.cc common.cc geometry.cc region.cc region_tr.cc
 * multigrid.cc) plus the single-rank MPI shim and the LAPACK stand-in.
 *
 * TEST INFRASTRUCTURE ONLY.  Tests load it through ctypes to (a) pin the C
 * restatement in oracle/pgmg_oracle.c against the reference itself and
 * (b) time the reference CPU path for the benchmark's reference arm.
 *
 * Every call goes through the reference's public API only:
 *   multigrid(p_class&,geometry&,comm_buffer&)   multigrid.hh:283-295
 *   setup_matrices / setup_fields                 multigrid.hh:302-319
 *   v_cycle, fmg_cycle                            multigrid.cc:88-134
 *   gauss_seidel(mode,level), restriction(level),
 *   interpolation(level), solve_exact(level)      multigrid.cc:180-224, multigrid.hh:265
 *   l2_error_all, rhs_l2norm                      multigrid.cc:246-261
 *   solve_v_cycles, guide.set_tol                 multigrid.hh:88-96, 182-219
 *   reg[l]->{x0,r0,S,A,mg,ng,m,n,o,Aexact}        region.hh:30-76, 252-398
 * and region::gs_num (region.cc:116) to count smoothing sweeps.
 */
#include <cstring>
#include <cstdlib>
#include <vector>

#include "multigrid.hh"

namespace {

/* A problem class (the duck-typed p_class concept, problem_simple.hh:36-73)
 * backed by caller-owned arrays: per-point box bounds S (6 ints, relative
 * offsets [xd,xu,yd,yu,zd,zu]) and 27-slot coefficients (slot
 * (di+1)+3(dj+1)+9(dk+1)), natural order i fastest.  Every point is
 * "internal", so the reference copies the box entries through
 * fill_entries (region.hh:96-101, 505, 512-516). */
struct array_problem {
	bool x_prd,y_prd,z_prd;
	int m,n,o;
	const int *S;
	const double *c27;
	const double *r;
	const double *x;
	inline long idx(int i,int j,int k) const {return i+(long)m*(j+(long)n*k);}
	inline int range_xd(int i,int j,int k) {return S[6*idx(i,j,k)];}
	inline int range_xu(int i,int j,int k) {return S[6*idx(i,j,k)+1];}
	inline int range_yd(int i,int j,int k) {return S[6*idx(i,j,k)+2];}
	inline int range_yu(int i,int j,int k) {return S[6*idx(i,j,k)+3];}
	inline int range_zd(int i,int j,int k) {return S[6*idx(i,j,k)+4];}
	inline int range_zu(int i,int j,int k) {return S[6*idx(i,j,k)+5];}
	inline bool internal(int,int,int) {return true;}
	inline int mem_size(int i,int j,int k) {
		const int *s=S+6*idx(i,j,k);
		return (s[1]-s[0])*(s[3]-s[2])*(s[5]-s[4]);
	}
	void fill_entries(int i,int j,int k,double *&en) {
		const int *s=S+6*idx(i,j,k);
		const double *c=c27+27*idx(i,j,k);
		for(int dk=s[4];dk<s[5];dk++) for(int dj=s[2];dj<s[3];dj++)
			for(int di=s[0];di<s[1];di++) *(en++)=c[(di+1)+3*(dj+1)+9*(dk+1)];
	}
	inline double* external_ptr(int,int,int) {return NULL;}
	inline double x_field(int i,int j,int k) {return x?x[idx(i,j,k)]:0.;}
	inline double r_field(int i,int j,int k) {return r?r[idx(i,j,k)]:0.;}
};

struct ref_handle {
	comm_buffer com;
	geometry *gm;
	array_problem pr;
	multigrid *mg;
	std::vector<double> r,x;
};

inline region* lev(ref_handle *h,int l) {return h->mg->reg[l];}

}

extern "C" {

/* Builds the reference hierarchy for an m x n x o grid and fills level 0
 * from the given arrays.  S and c27 are read during this call only (the
 * reference copies the entries into its own storage); r and x are copied and
 * may be NULL (zero fields). */
void* ref_create(int m,int n,int o,int xp,int yp,int zp,const int *S,
		 const double *c27,const double *r,const double *x) {
	ref_handle *h=new ref_handle;
	long N=(long)m*n*o;
	h->r.assign(N,0.);h->x.assign(N,0.);
	if(r) memcpy(&h->r[0],r,N*sizeof(double));
	if(x) memcpy(&h->x[0],x,N*sizeof(double));
	h->gm=new geometry(m,n,o,xp!=0,yp!=0,zp!=0);
	array_problem &p=h->pr;
	p.x_prd=xp!=0;p.y_prd=yp!=0;p.z_prd=zp!=0;
	p.m=m;p.n=n;p.o=o;
	p.S=S;p.c27=c27;p.r=&h->r[0];p.x=&h->x[0];
	h->mg=new multigrid(p,*h->gm,h->com);
	h->mg->setup_matrices(p);
	h->mg->setup_fields(p);
	p.S=NULL;p.c27=NULL;
	return h;
}

void ref_destroy(void *hv) {
	ref_handle *h=static_cast<ref_handle*>(hv);
	delete h->mg;
	h->gm->free();
	delete h->gm;
	delete h;
}

int ref_nlevels(void *hv) {return static_cast<ref_handle*>(hv)->mg->mlevels;}

void ref_level_dims(void *hv,int l,int *mno) {
	region *g=lev(static_cast<ref_handle*>(hv),l);
	mno[0]=g->m;mno[1]=g->n;mno[2]=g->o;
}

/* 1 if the bottom level solves with the LU factorisation, 0 if the reference
 * fell back to 24 Gauss-Seidel sweeps (region_tr.cc:524-533, :557). */
int ref_lu_enabled(void *hv) {
	ref_handle *h=static_cast<ref_handle*>(hv);
	return lev(h,h->mg->mlevels-1)->Aexact!=NULL?1:0;
}

void ref_get_x(void *hv,int l,double *out) {
	region *g=lev(static_cast<ref_handle*>(hv),l);
	for(int k=0;k<g->so;k++) for(int j=0;j<g->sn;j++) for(int i=0;i<g->sm;i++)
		*(out++)=g->x0[i+g->mg*(j+g->ng*k)];
}

void ref_set_x(void *hv,int l,const double *in) {
	region *g=lev(static_cast<ref_handle*>(hv),l);
	for(int k=0;k<g->so;k++) for(int j=0;j<g->sn;j++) for(int i=0;i<g->sm;i++)
		g->x0[i+g->mg*(j+g->ng*k)]=*(in++);
}

void ref_get_r(void *hv,int l,double *out) {
	region *g=lev(static_cast<ref_handle*>(hv),l);
	memcpy(out,g->r0,sizeof(double)*g->smno);
}

void ref_set_r(void *hv,int l,const double *in) {
	region *g=lev(static_cast<ref_handle*>(hv),l);
	memcpy(g->r0,in,sizeof(double)*g->smno);
}

void ref_get_S(void *hv,int l,int *out) {
	region *g=lev(static_cast<ref_handle*>(hv),l);
	memcpy(out,g->S,sizeof(int)*6*g->smno);
}

/* Expands the level's box-stored coefficients into 27 slots.  Returns the
 * number of points whose box does not fit in [-1,2)^3 (those are skipped). */
int ref_get_A27(void *hv,int l,double *out) {
	region *g=lev(static_cast<ref_handle*>(hv),l);
	int bad=0;
	memset(out,0,sizeof(double)*27*(size_t)g->smno);
	for(int q=0;q<g->smno;q++) {
		const int *s=g->S+6*q;
		const double *a=g->A[q];
		double *o=out+27*(size_t)q;
		if(s[0]<-1||s[1]>2||s[2]<-1||s[3]>2||s[4]<-1||s[5]>2) {bad++;continue;}
		for(int dk=s[4];dk<s[5];dk++) for(int dj=s[2];dj<s[3];dj++)
			for(int di=s[0];di<s[1];di++) o[(di+1)+3*(dj+1)+9*(dk+1)]=*(a++);
	}
	return bad;
}

void ref_gauss_seidel(void *hv,int mode,int l) {static_cast<ref_handle*>(hv)->mg->gauss_seidel(mode,l);}
void ref_restriction(void *hv,int l) {static_cast<ref_handle*>(hv)->mg->restriction(l);}
void ref_interpolation(void *hv,int l) {static_cast<ref_handle*>(hv)->mg->interpolation(l);}
void ref_solve_exact(void *hv,int l) {static_cast<ref_handle*>(hv)->mg->solve_exact(l);}
void ref_v_cycle(void *hv,int mode) {static_cast<ref_handle*>(hv)->mg->v_cycle(mode);}
void ref_fmg_cycle(void *hv) {static_cast<ref_handle*>(hv)->mg->fmg_cycle();}
double ref_l2_error_all(void *hv,int l) {return static_cast<ref_handle*>(hv)->mg->l2_error_all(l);}
double ref_rhs_l2norm(void *hv,int l) {return static_cast<ref_handle*>(hv)->mg->rhs_l2norm(l);}
void ref_setup_test(void *hv,int ca,int xfield,int l) {static_cast<ref_handle*>(hv)->mg->setup_test(ca,xfield!=0,l);}
void ref_clear_x(void *hv,int l) {lev(static_cast<ref_handle*>(hv),l)->clear_x_field();}

/* Runs multigrid::solve_v_cycles with guide.set_tol(p_scale) (set once, on
 * the first call).  Returns its status (0 converged, 1 cap, 2 NaN); the
 * squared residual goes to *res and the number of Gauss-Seidel sweeps the
 * call performed to *sweeps (region::gs_num, region.cc:116). */
int ref_solve_v_cycles(void *hv,double p_scale,double *res,long *sweeps) {
	ref_handle *h=static_cast<ref_handle*>(hv);
	if(!h->mg->guide.tol_set_manually) h->mg->guide.set_tol(p_scale);
	int g0=region::gs_num;
	int st=h->mg->solve_v_cycles(*res);
	*sweeps=region::gs_num-g0;
	return st;
}

/* The reference's PCG helpers on level 0 (region.cc:1848-1940,
 * region.hh:226-236, multigrid.hh:222-251); arrays in natural order (on one
 * non-periodic process the reference's x layout is natural order). */
void ref_compute_residual(void *hv,double *out) {static_cast<ref_handle*>(hv)->mg->compute_residual(out);}
void ref_Ax(void *hv,const double *in,double *out) {static_cast<ref_handle*>(hv)->mg->Ax(in,out);}
void ref_unpadded_Ax(void *hv,const double *in,double *out) {static_cast<ref_handle*>(hv)->mg->unpadded_Ax(in,out);}
double ref_source_soln_dot(void *hv) {return static_cast<ref_handle*>(hv)->mg->source_soln_dot();}
double ref_soln_diff(void *hv,double *ext_x) {return static_cast<ref_handle*>(hv)->mg->soln_diff(ext_x);}
void ref_copy_rhs_to_soln(void *hv) {static_cast<ref_handle*>(hv)->mg->copy_rhs_to_soln();}
double ref_l0_error_all(void *hv,int l) {return static_cast<ref_handle*>(hv)->mg->l0_error_all(l);}

int ref_guide_pred_iters(void *hv) {return static_cast<ref_handle*>(hv)->mg->guide.pred_iters();}

long ref_gs_count() {return region::gs_num;}

}
