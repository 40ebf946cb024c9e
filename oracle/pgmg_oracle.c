/* CPU restatement of the PGMG reference multigrid hot path (oracle).
 *
 * TEST INFRASTRUCTURE ONLY -- the checker, never the thing measured or
 * shipped.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it.
 *
 * Restated from the reference for one process and non-periodic axes; every
 * routine names the reference lines it follows.  Arithmetic is FP64 without
 * fused multiply-add (built with -ffp-contract=off), and every accumulation
 * runs in the reference's order, so results match the reference bit for bit
 * (checked against oracle/_ref/libpgmg_ref.so by tests/test_oracle_pin.py).
 *
 * Layout: 27 slots per point, slot (di+1)+3(dj+1)+9(dk+1), zero outside the
 * point's box; boxes as 6 ints [xd,xu,yd,yu,zd,zu] relative to the point
 * (region.hh:252-256); x stored with a one-point zero halo so that every
 * slot can be read; r dense (region.hh:55).
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "pgmg_oracle.h"

#define ORC_MAXL 16          /* mg_max_levels, common.hh:15 */
#define ORC_GS_EXACT 24      /* pgmg_gs_exact, common.hh:62 */
#define ORC_MAX_EXACT 2048   /* pgmg_max_exact, common.hh:65 */

typedef struct {
	int m,n,o;
	long N;
	double *A;   /* 27*N */
	int *S;      /* 6*N  */
	double *x;   /* (m+2)(n+2)(o+2) */
	double *r;   /* N */
} olev;

struct orc {
	int nl;
	olev L[ORC_MAXL];
	int lu_ok;
	double *LU;
	int *piv;
	double *buf;
	long gs_num;
	/* multigrid::mg_guide state, multigrid.hh:34-118 */
	int period,iter,use_avg,tol_set;
	double iter_avg,iter_var,alpha,tol;
	int v_down,v_up,v_bottom;
	int smoother;  /* 0 = lexicographic (reference), 1 = 8-colour */
	long long slab_budget;  /* bytes of FP64 x per z-slab of the 8-colour sweep */
};

static inline long xi(const olev *L,int i,int j,int k) {
	return (i+1)+(long)(L->m+2)*((j+1)+(long)(L->n+2)*(k+1));
}
static inline long pi(const olev *L,int i,int j,int k) {
	return i+(long)L->m*(j+(long)L->n*k);
}

/* Per-axis cube geometry of the transfer between a fine axis of size ma and
 * its coarse axis sm=(ma+2)>>1 (region.cc:14), following rt_scan_grid /
 * rt_scan_slice / rt_scan_row (region.cc:665-746) on one rank (ai=0,
 * bi=ma): cubes C = 0..last; the lower point 2C always exists; the upper
 * point 2C+1 exists unless C is the last cube of an odd axis; on an even
 * axis the last cube's upper point (ma-1) "snaps" onto coarse C+1 with
 * weight 1 (mask bits 4/32/256). */
static inline int cube_last(int ma) {int sm=(ma+2)>>1;return (ma&1)?sm-1:sm-2;}
static inline int has_upper(int C,int ma) {return 2*C+1<ma;}
static inline int snapped(int C,int ma) {return !(ma&1)&&C==cube_last(ma);}

/* grid_map, non-periodic branch (region.cc:1209-1216). */
static void grid_map(int *lo,int *hi,int ma) {
	*lo=(!(ma&1)&&*lo==ma-1?*lo+1:*lo)>>1;
	*hi=(*hi+2)>>1;
}

/* igrid_map, non-periodic branch with the crop to the stencil box
 * (region.cc:1243-1258). */
static int igrid_map(int *lo,int *hi,int blo,int bhi,int i,int ma) {
	int j=i<<1;
	if(ma&1) {*lo=j==0?0:j-1;*hi=j==ma-1?ma:j+2;}
	else {
		if(j==ma) {*lo=ma-1;*hi=ma;j=ma-1;}
		else {*lo=j==0?0:j-1;*hi=j==ma-2?ma-1:j+2;}
	}
	if(*lo<blo) *lo=blo;
	if(*hi>bhi) *hi=bhi;
	return j;
}

static void level_alloc(olev *L,int m,int n,int o) {
	L->m=m;L->n=n;L->o=o;L->N=(long)m*n*o;
	L->A=calloc(27*L->N,sizeof(double));
	L->S=calloc(6*L->N,sizeof(int));
	L->x=calloc((size_t)(m+2)*(n+2)*(o+2),sizeof(double));
	L->r=calloc(L->N,sizeof(double));
}

/* region::residual (region.cc:1833-1842): r - sum over the box, box order. */
static double residual(const olev *L,int i,int j,int k) {
	const double *a=L->A+27*pi(L,i,j,k);
	double Ax=0;
	for(int dk=0;dk<3;dk++) for(int dj=0;dj<3;dj++) for(int di=0;di<3;di++)
		Ax+=a[di+3*dj+9*dk]*L->x[xi(L,i+di-1,j+dj-1,k+dk-1)];
	return L->r[pi(L,i,j,k)]-Ax;
}

/* One point of region::gauss_seidel (region.cc:367-446): terms in box order
 * with the centre skipped, then x=(r-Ax)*(1/centre). */
static inline void gs_point(olev *L,int i,int j,int k) {
	const double *a=L->A+27*pi(L,i,j,k);
	double Ax=0;
	for(int q=0;q<27;q++) {
		if(q==13) continue;
		int di=q%3-1,dj=(q/3)%3-1,dk=q/9-1;
		Ax+=a[q]*L->x[xi(L,i+di,j+dj,k+dk)];
	}
	double Axc=1./a[13];
	L->x[xi(L,i,j,k)]=(L->r[pi(L,i,j,k)]-Ax)*Axc;
}

/* fill_rat_bounds (region.cc:598-623) with rat_bound_full/partial
 * (:916-1003), b_red (:1105-1110), Sbound (:1266-1271), b_ex (:1276-1283):
 * each coarse box starts as [0,1)^3 and is extended by the grid_map'ed
 * global box of every fine point that transfers to it. */
static void rat_bounds(const olev *F,olev *Cl) {
	for(long q=0;q<Cl->N;q++) {
		int *s=Cl->S+6*q;
		s[0]=s[2]=s[4]=0;s[1]=s[3]=s[5]=1;
	}
	int lx=cube_last(F->m),ly=cube_last(F->n),lz=cube_last(F->o);
	for(int Cz=0;Cz<=lz;Cz++) for(int Cy=0;Cy<=ly;Cy++) for(int Cx=0;Cx<=lx;Cx++)
	for(int dz=0;dz<2;dz++) for(int dy=0;dy<2;dy++) for(int dx=0;dx<2;dx++) {
		if((dx&&!has_upper(Cx,F->m))||(dy&&!has_upper(Cy,F->n))||(dz&&!has_upper(Cz,F->o))) continue;
		int ti=2*Cx+dx,tj=2*Cy+dy,tk=2*Cz+dz;
		const int *fs=F->S+6*pi(F,ti,tj,tk);
		int St[6]={fs[0]+ti,fs[1]+ti,fs[2]+tj,fs[3]+tj,fs[4]+tk,fs[5]+tk};
		grid_map(St,St+1,F->m);grid_map(St+2,St+3,F->n);grid_map(St+4,St+5,F->o);
		int tx[2],ty[2],tz[2],nx=0,ny=0,nz=0;
		if(!dx) tx[nx++]=Cx; else if(snapped(Cx,F->m)) tx[nx++]=Cx+1; else {tx[nx++]=Cx;tx[nx++]=Cx+1;}
		if(!dy) ty[ny++]=Cy; else if(snapped(Cy,F->n)) ty[ny++]=Cy+1; else {ty[ny++]=Cy;ty[ny++]=Cy+1;}
		if(!dz) tz[nz++]=Cz; else if(snapped(Cz,F->o)) tz[nz++]=Cz+1; else {tz[nz++]=Cz;tz[nz++]=Cz+1;}
		for(int c=0;c<nz;c++) for(int b=0;b<ny;b++) for(int a=0;a<nx;a++) {
			int I=tx[a],J=ty[b],K=tz[c];
			int *s=Cl->S+6*pi(Cl,I,J,K);
			if(St[0]-I<s[0]) s[0]=St[0]-I;
			if(St[1]-I>s[1]) s[1]=St[1]-I;
			if(St[2]-J<s[2]) s[2]=St[2]-J;
			if(St[3]-J>s[3]) s[3]=St[3]-J;
			if(St[4]-K<s[4]) s[4]=St[4]-K;
			if(St[5]-K>s[5]) s[5]=St[5]-K;
		}
	}
}

/* compute_rats (region.cc:629-660): for every fine point, in cube scan
 * order, A_red (:1117-1166) forms the row 0.125*sum_u A(t,u)*w(u->J) over
 * J in the grid_map'ed box, with u in igrid_map's range cropped to the
 * point's box and w = 1 or 1/2 per axis (kfac/jkfac, :1154-1159); A_mul /
 * A_sca (region.hh:460-465) scale it by 1/2 per non-snapped upper axis; A_add
 * (:1173-1180) adds it to every coarse corner the point transfers to. */
static void rat_fill(const olev *F,olev *Cl) {
	memset(Cl->A,0,sizeof(double)*27*Cl->N);
	double At[27];
	int lx=cube_last(F->m),ly=cube_last(F->n),lz=cube_last(F->o);
	for(int Cz=0;Cz<=lz;Cz++) for(int Cy=0;Cy<=ly;Cy++) for(int Cx=0;Cx<=lx;Cx++)
	for(int dz=0;dz<2;dz++) for(int dy=0;dy<2;dy++) for(int dx=0;dx<2;dx++) {
		if((dx&&!has_upper(Cx,F->m))||(dy&&!has_upper(Cy,F->n))||(dz&&!has_upper(Cz,F->o))) continue;
		int ti=2*Cx+dx,tj=2*Cy+dy,tk=2*Cz+dz;
		const int *fs=F->S+6*pi(F,ti,tj,tk);
		const double *fa=F->A+27*pi(F,ti,tj,tk);
		int B[6]={fs[0]+ti,fs[1]+ti,fs[2]+tj,fs[3]+tj,fs[4]+tk,fs[5]+tk};
		int St[6]={B[0],B[1],B[2],B[3],B[4],B[5]};
		grid_map(St,St+1,F->m);grid_map(St+2,St+3,F->n);grid_map(St+4,St+5,F->o);
		int sx=St[1]-St[0],sy=St[3]-St[2];
		double *Ap=At;
		for(int vk=St[4];vk<St[5];vk++) {
			int lk,uk,ck=igrid_map(&lk,&uk,B[4],B[5],vk,F->o);
			for(int vj=St[2];vj<St[3];vj++) {
				int lj,uj,cj=igrid_map(&lj,&uj,B[2],B[3],vj,F->n);
				for(int vi=St[0];vi<St[1];vi++,Ap++) {
					int li,ui,ci=igrid_map(&li,&ui,B[0],B[1],vi,F->m);
					*Ap=0;
					for(int kk=lk;kk<uk;kk++) {
						double kfac=kk==ck?1:0.5;
						for(int jj=lj;jj<uj;jj++) {
							double jkfac=jj==cj?kfac:0.5*kfac;
							for(int ii=li;ii<ui;ii++)
								*Ap+=0.125*fa[(ii-ti+1)+3*(jj-tj+1)+9*(kk-tk+1)]
								    *(ii==ci?jkfac:0.5*jkfac);
						}
					}
				}
			}
		}
		int nAt=(int)(Ap-At);
		double fac=(dx&&!snapped(Cx,F->m)?0.5:1)*(dy&&!snapped(Cy,F->n)?0.5:1)*(dz&&!snapped(Cz,F->o)?0.5:1);
		if(fac!=1) for(int q=0;q<nAt;q++) At[q]*=fac;
		int tx[2],ty[2],tz[2],nx=0,ny=0,nz=0;
		if(!dx) tx[nx++]=Cx; else if(snapped(Cx,F->m)) tx[nx++]=Cx+1; else {tx[nx++]=Cx;tx[nx++]=Cx+1;}
		if(!dy) ty[ny++]=Cy; else if(snapped(Cy,F->n)) ty[ny++]=Cy+1; else {ty[ny++]=Cy;ty[ny++]=Cy+1;}
		if(!dz) tz[nz++]=Cz; else if(snapped(Cz,F->o)) tz[nz++]=Cz+1; else {tz[nz++]=Cz;tz[nz++]=Cz+1;}
		for(int c=0;c<nz;c++) for(int b=0;b<ny;b++) for(int a=0;a<nx;a++) {
			int I=tx[a],J=ty[b],K=tz[c];
			double *ca=Cl->A+27*pi(Cl,I,J,K);
			const double *atp=At;
			for(int vk=St[4];vk<St[5];vk++) for(int vj=St[2];vj<St[3];vj++)
				for(int vi=St[0];vi<St[1];vi++)
					ca[(vi-I+1)+3*(vj-J+1)+9*(vk-K+1)]+=*(atp++);
		}
		(void)sx;(void)sy;
	}
}

/* lu_decomposition (region_tr.cc:483-534): dense column-major matrix
 * Aexact[row+col*n], LU with partial pivoting, then the conditioning check
 * |U_nn|/|U_11| < eps*1e4 (common.hh:58) that switches to Gauss-Seidel. */
static void lu_setup(orc *h) {
	olev *L=&h->L[h->nl-1];
	int n=(int)L->N;
	free(h->LU);free(h->piv);free(h->buf);
	h->LU=NULL;h->piv=NULL;h->buf=NULL;h->lu_ok=0;
	if(n>=ORC_MAX_EXACT) return;
	h->LU=calloc((size_t)n*n,sizeof(double));
	h->piv=calloc(n,sizeof(int));
	h->buf=calloc(n,sizeof(double));
	for(int k=0;k<L->o;k++) for(int j=0;j<L->n;j++) for(int i=0;i<L->m;i++) {
		long row=pi(L,i,j,k);
		const double *a=L->A+27*row;
		for(int q=0;q<27;q++) {
			int di=q%3-1,dj=(q/3)%3-1,dk=q/9-1;
			int ii=i+di,jj=j+dj,kk=k+dk;
			if(ii<0||jj<0||kk<0||ii>=L->m||jj>=L->n||kk>=L->o) continue;
			h->LU[row+(size_t)pi(L,ii,jj,kk)*n]=a[q];
		}
	}
	int info=orc_dgetrf(n,h->LU,h->piv);
	double hi=fabs(h->LU[0]),lo=fabs(h->LU[(size_t)n*n-1]);
	if(info!=0||hi==0||lo/hi<DBL_EPSILON*1e4) {
		free(h->LU);free(h->piv);free(h->buf);
		h->LU=NULL;h->piv=NULL;h->buf=NULL;
	} else h->lu_ok=1;
}

int orc_dgetrf(int n,double *a,int *ipiv) {
	int info=0;
	for(int j=0;j<n;j++) {
		int p=j;
		double best=fabs(a[j+(size_t)j*n]);
		for(int i=j+1;i<n;i++) {
			double v=fabs(a[i+(size_t)j*n]);
			if(v>best) {best=v;p=i;}
		}
		ipiv[j]=p+1;
		if(a[p+(size_t)j*n]!=0.0) {
			if(p!=j) for(int k=0;k<n;k++) {
				double t=a[j+(size_t)k*n];a[j+(size_t)k*n]=a[p+(size_t)k*n];a[p+(size_t)k*n]=t;
			}
			double r=1.0/a[j+(size_t)j*n];
			for(int i=j+1;i<n;i++) a[i+(size_t)j*n]*=r;
		} else if(info==0) info=j+1;
		for(int k=j+1;k<n;k++) {
			double u=a[j+(size_t)k*n];
			if(u!=0.0) for(int i=j+1;i<n;i++) a[i+(size_t)k*n]-=a[i+(size_t)j*n]*u;
		}
	}
	return info;
}

void orc_dgetrs(int n,const double *a,const int *ipiv,double *x) {
	for(int i=0;i<n;i++) {
		int p=ipiv[i]-1;
		if(p!=i) {double t=x[i];x[i]=x[p];x[p]=t;}
	}
	for(int j=0;j<n;j++) {
		double xj=x[j];
		if(xj!=0.0) for(int i=j+1;i<n;i++) x[i]-=xj*a[i+(size_t)j*n];
	}
	for(int j=n-1;j>=0;j--) {
		if(x[j]!=0.0) {
			x[j]/=a[j+(size_t)j*n];
			double xj=x[j];
			for(int i=0;i<j;i++) x[i]-=xj*a[i+(size_t)j*n];
		}
	}
}

orc* orc_create(int m,int n,int o,const int *S6,const double *c27,const double *r,
		const double *x,int coarse) {
	orc *h=calloc(1,sizeof(orc));
	/* multigrid ctor defaults, multigrid.hh:283-285 */
	h->v_down=2;h->v_bottom=20;h->v_up=2;
	h->slab_budget=0;
	/* mg_guide(), multigrid.hh:79-82, set_period :107-111 */
	h->period=16;h->iter=16;h->iter_avg=16;h->iter_var=1000000;h->alpha=3.0/16;
	level_alloc(&h->L[0],m,n,o);
	olev *L0=&h->L[0];
	memcpy(L0->S,S6,sizeof(int)*6*L0->N);
	memcpy(L0->A,c27,sizeof(double)*27*L0->N);
	if(r) memcpy(L0->r,r,sizeof(double)*L0->N);
	if(x) for(int k=0;k<o;k++) for(int j=0;j<n;j++) for(int i=0;i<m;i++)
		L0->x[xi(L0,i,j,k)]=x[pi(L0,i,j,k)];
	/* setup_hierarchy, multigrid.cc:17-85: coarsen while m*n*o > 1024,
	 * m_c = (m+2)>>1 on non-periodic axes (region.cc:14). */
	h->nl=1;
	while((long)h->L[h->nl-1].m*h->L[h->nl-1].n*h->L[h->nl-1].o>1024&&h->nl<ORC_MAXL) {
		olev *F=&h->L[h->nl-1];
		level_alloc(&h->L[h->nl],(F->m+2)>>1,(F->n+2)>>1,(F->o+2)>>1);
		rat_bounds(F,&h->L[h->nl]);
		h->nl++;
	}
	/* multigrid::compute_rats, multigrid.cc:138-152, then the bottom LU. */
	for(int l=1;l<h->nl;l++) rat_fill(&h->L[l-1],&h->L[l]);
	if(coarse) lu_setup(h);
	return h;
}

void orc_destroy(orc *h) {
	for(int l=0;l<h->nl;l++) {free(h->L[l].A);free(h->L[l].S);free(h->L[l].x);free(h->L[l].r);}
	free(h->LU);free(h->piv);free(h->buf);
	free(h);
}

int orc_nlevels(orc *h) {return h->nl;}
void orc_level_dims(orc *h,int l,int *mno) {mno[0]=h->L[l].m;mno[1]=h->L[l].n;mno[2]=h->L[l].o;}
int orc_lu_enabled(orc *h) {return h->lu_ok;}

void orc_get_x(orc *h,int l,double *out) {
	olev *L=&h->L[l];
	for(int k=0;k<L->o;k++) for(int j=0;j<L->n;j++) for(int i=0;i<L->m;i++) *(out++)=L->x[xi(L,i,j,k)];
}
void orc_set_x(orc *h,int l,const double *in) {
	olev *L=&h->L[l];
	for(int k=0;k<L->o;k++) for(int j=0;j<L->n;j++) for(int i=0;i<L->m;i++) L->x[xi(L,i,j,k)]=*(in++);
}
void orc_get_r(orc *h,int l,double *out) {memcpy(out,h->L[l].r,sizeof(double)*h->L[l].N);}
void orc_set_r(orc *h,int l,const double *in) {memcpy(h->L[l].r,in,sizeof(double)*h->L[l].N);}
void orc_get_S(orc *h,int l,int *out) {memcpy(out,h->L[l].S,sizeof(int)*6*h->L[l].N);}
void orc_get_A27(orc *h,int l,double *out) {memcpy(out,h->L[l].A,sizeof(double)*27*h->L[l].N);}

/* region::gauss_seidel (region.cc:355-542): forward lexicographic sweep,
 * plus the full backward sweep when mode != 0. */
void orc_gauss_seidel(orc *h,int mode,int l) {
	olev *L=&h->L[l];
	h->gs_num++;
	for(int k=0;k<L->o;k++) for(int j=0;j<L->n;j++) for(int i=0;i<L->m;i++) gs_point(L,i,j,k);
	if(!mode) return;
	for(int k=L->o-1;k>=0;k--) for(int j=L->n-1;j>=0;j--) for(int i=L->m-1;i>=0;i--) gs_point(L,i,j,k);
}

/* Colour order of the library's 8-colour sweep: the colours with i+j+k
 * even first (000, 011, 101, 110 as (i&1,j&1,k&1)), then the odd ones (111,
 * 100, 010, 001). */
static const int colour_seq[8]={0,6,5,3,7,1,2,4};

/* The 8-colour smoother of this library (not in the reference): colour
 * c = (i&1)|(j&1)<<1|(k&1)<<2 in the order colour_seq (reversed for the
 * backward half of mode != 0); points of one colour are independent for a
 * 27-point box. */
void orc_gauss_seidel_mc8(orc *h,int mode,int l) {
	olev *L=&h->L[l];
	h->gs_num++;
	/* Slab blocking: a level whose FP64 solution array (with its one-point
	 * halo) exceeds slab_budget bytes is swept in z-slabs of colour planes,
	 * all 8 colours of a slab before the next; slab s covers colour planes
	 * k2 in [O2*s/S, O2*(s+1)/S). */
	int O2=(L->o+1)/2,S=1;
	long long xb=(long long)(L->m+2)*(L->n+2)*(L->o+2)*8;
	if(h->slab_budget>0&&xb>h->slab_budget) {
		long long q=(xb+h->slab_budget-1)/h->slab_budget;
		S=(int)(q<O2?q:O2);
	}
	for(int pass=0;pass<(mode?2:1);pass++)
	for(int ss=0;ss<S;ss++) {
		int sl=pass?S-1-ss:ss;
		int k2lo=(int)((long long)O2*sl/S),k2hi=(int)((long long)O2*(sl+1)/S);
		for(int cc=0;cc<8;cc++) {
			int c=colour_seq[pass?7-cc:cc];
			int a=c&1,b=(c>>1)&1,e=(c>>2)&1;
			for(int k2=k2lo;k2<k2hi;k2++) {
				int k=2*k2+e;
				if(k>=L->o) continue;
				for(int j=b;j<L->n;j+=2) for(int i=a;i<L->m;i+=2) gs_point(L,i,j,k);
			}
		}
	}
}

void orc_set_slab_budget(orc *h,long long bytes) {h->slab_budget=bytes;}


/* region::restriction (region.cc:546-572) with restrict_full/partial
 * (:818-912): clear the coarse r, then for each fine point in cube scan
 * order add 0.125*w*residual to every coarse corner it transfers to
 * (w = 1/2 per non-snapped upper axis).  multigrid::restriction then clears
 * the coarse x (multigrid.cc:219). */
void orc_restriction(orc *h,int l) {
	olev *F=&h->L[l-1],*Cl=&h->L[l];
	memset(Cl->r,0,sizeof(double)*Cl->N);
	int lx=cube_last(F->m),ly=cube_last(F->n),lz=cube_last(F->o);
	for(int Cz=0;Cz<=lz;Cz++) for(int Cy=0;Cy<=ly;Cy++) for(int Cx=0;Cx<=lx;Cx++)
	for(int dz=0;dz<2;dz++) for(int dy=0;dy<2;dy++) for(int dx=0;dx<2;dx++) {
		if((dx&&!has_upper(Cx,F->m))||(dy&&!has_upper(Cy,F->n))||(dz&&!has_upper(Cz,F->o))) continue;
		double res=residual(F,2*Cx+dx,2*Cy+dy,2*Cz+dz);
		/* restrict_partial tests the x snap flag for the y axis of the
		 * (ti,tj+1,tk+1) point (region.cc:888-895: "if(xs) v6+=rd" where
		 * the other roles test ys); it differs from P^T only on
		 * even-sized axes and is reproduced here as the reference does it. */
		int ysn=(!dx&&dy&&dz)?snapped(Cx,F->m):snapped(Cy,F->n);
		double fac=0.125*(dx&&!snapped(Cx,F->m)?0.5:1)*(dy&&!ysn?0.5:1)*(dz&&!snapped(Cz,F->o)?0.5:1);
		double rd=fac*res;
		int tx[2],ty[2],tz[2],nx=0,ny=0,nz=0;
		if(!dx) tx[nx++]=Cx; else if(snapped(Cx,F->m)) tx[nx++]=Cx+1; else {tx[nx++]=Cx;tx[nx++]=Cx+1;}
		if(!dy) ty[ny++]=Cy; else if(ysn) ty[ny++]=Cy+1; else {ty[ny++]=Cy;ty[ny++]=Cy+1;}
		if(!dz) tz[nz++]=Cz; else if(snapped(Cz,F->o)) tz[nz++]=Cz+1; else {tz[nz++]=Cz;tz[nz++]=Cz+1;}
		for(int c=0;c<nz;c++) for(int b=0;b<ny;b++) for(int a=0;a<nx;a++)
			Cl->r[pi(Cl,tx[a],ty[b],tz[c])]+=rd;
	}
	orc_clear_x(h,l);
}

/* region::interpolation (region.cc:576-593): interpolate_full (:752-772)
 * on interior cubes, interpolate_partial (:779-810) on the last cube of any
 * row, row or slice; the two differ in how some sums associate. */
void orc_interpolation(orc *h,int l) {
	olev *F=&h->L[l-1],*Cl=&h->L[l];
	int lx=cube_last(F->m),ly=cube_last(F->n),lz=cube_last(F->o);
	for(int Cz=0;Cz<=lz;Cz++) for(int Cy=0;Cy<=ly;Cy++) for(int Cx=0;Cx<=lx;Cx++) {
		int ux=has_upper(Cx,F->m),uy=has_upper(Cy,F->n),uz=has_upper(Cz,F->o);
		double v[8];
		for(int q=0;q<8;q++) {
			int a=q&1,b=(q>>1)&1,c=q>>2;
			int I=Cx+a,J=Cy+b,K=Cz+c;
			v[q]=(I<Cl->m&&J<Cl->n&&K<Cl->o)?Cl->x[xi(Cl,I,J,K)]:-99.;
		}
		double *x=F->x;
		int ti=2*Cx,tj=2*Cy,tk=2*Cz;
		if(Cx<lx&&Cy<ly&&Cz<lz) {
			double t1,t2,t3;
			x[xi(F,ti,tj,tk)]+=v[0];
			x[xi(F,ti+1,tj,tk)]+=0.5*(t1=v[0]+v[1]);
			x[xi(F,ti,tj+1,tk)]+=0.5*(v[0]+v[2]);
			x[xi(F,ti+1,tj+1,tk)]+=0.25*(t2=t1+v[2]+v[3]);
			x[xi(F,ti,tj,tk+1)]+=0.5*(v[0]+v[4]);
			x[xi(F,ti+1,tj,tk+1)]+=0.25*(t1+(t3=v[4]+v[5]));
			x[xi(F,ti,tj+1,tk+1)]+=0.25*(v[0]+v[2]+v[4]+v[6]);
			x[xi(F,ti+1,tj+1,tk+1)]+=0.125*(t2+t3+v[6]+v[7]);
		} else {
			int xs=snapped(Cx,F->m),ys=snapped(Cy,F->n),zs=snapped(Cz,F->o);
			double t2=0,t3;
			x[xi(F,ti,tj,tk)]+=v[0];
			if(ux) x[xi(F,ti+1,tj,tk)]+=xs?v[1]:0.5*(v[0]+v[1]);
			if(uy) x[xi(F,ti,tj+1,tk)]+=ys?v[2]:0.5*(v[0]+v[2]);
			if(uz) x[xi(F,ti,tj,tk+1)]+=zs?v[4]:0.5*(v[0]+v[4]);
			if(ux&&uz) x[xi(F,ti+1,tj,tk+1)]+=zs?(xs?v[5]:0.5*(v[4]+v[5])):(xs?0.5*(v[1]+v[5]):0.25*(v[0]+v[1]+v[4]+v[5]));
			if(uy&&uz) x[xi(F,ti,tj+1,tk+1)]+=zs?(ys?v[6]:0.5*(v[4]+v[6])):(ys?0.5*(v[2]+v[6]):0.25*(v[0]+v[2]+v[4]+v[6]));
			if(ux&&uy) {
				t2=ys?(xs?v[3]:0.5*(v[2]+v[3])):(xs?0.5*(v[1]+v[3]):0.25*(v[0]+v[1]+v[2]+v[3]));
				x[xi(F,ti+1,tj+1,tk)]+=t2;
				if(uz) {
					t3=ys?(xs?v[7]:0.5*(v[6]+v[7])):(xs?0.5*(v[5]+v[7]):0.25*(v[4]+v[5]+v[6]+v[7]));
					x[xi(F,ti+1,tj+1,tk+1)]+=zs?t3:0.5*(t3+t2);
				}
			}
		}
	}
}

static void gs_any(orc *h,int mode,int l) {
	if(h->smoother) orc_gauss_seidel_mc8(h,mode,l); else orc_gauss_seidel(h,mode,l);
}

void orc_set_smoother(orc *h,int mc8) {h->smoother=mc8?1:0;}

/* region::solve_exact (region_tr.cc:540-558): LU solve if enabled, else
 * pgmg_gs_exact plain sweeps (of the selected smoother). */
void orc_solve_exact(orc *h,int l) {
	olev *L=&h->L[l];
	if(l==h->nl-1&&h->lu_ok) {
		memcpy(h->buf,L->r,sizeof(double)*L->N);
		orc_dgetrs((int)L->N,h->LU,h->piv,h->buf);
		const double *p=h->buf;
		for(int k=0;k<L->o;k++) for(int j=0;j<L->n;j++) for(int i=0;i<L->m;i++) L->x[xi(L,i,j,k)]=*(p++);
	} else for(int q=0;q<ORC_GS_EXACT;q++) gs_any(h,0,l);
}

/* multigrid::v_cycle (multigrid.cc:88-106). */
void orc_v_cycle(orc *h,int mode) {
	int i,q,ml=h->nl;
	for(i=0;i<ml-1;i++) {
		for(q=0;q<h->v_down+i;q++) gs_any(h,mode,i);
		orc_restriction(h,i+1);
	}
	orc_solve_exact(h,ml-1);
	for(i=ml-1;i>0;i--) {
		orc_interpolation(h,i);
		for(q=0;q<h->v_up+i-1;q++) gs_any(h,mode,i-1);
	}
}

/* region::l2_error_all (region.cc:1475-1490): sum of squared residuals. */
double orc_l2_error_all(orc *h,int l) {
	olev *L=&h->L[l];
	double err=0;
	for(int k=0;k<L->o;k++) for(int j=0;j<L->n;j++) for(int i=0;i<L->m;i++) {
		double rem=residual(L,i,j,k);
		err+=rem*rem;
	}
	return err;
}

/* region::rhs_l2norm (region.cc:1549-1558). */
double orc_rhs_l2norm(orc *h,int l) {
	olev *L=&h->L[l];
	double s=0;
	for(long q=0;q<L->N;q++) s+=L->r[q]*L->r[q];
	return s;
}

void orc_clear_x(orc *h,int l) {
	olev *L=&h->L[l];
	for(int k=0;k<L->o;k++) for(int j=0;j<L->n;j++) for(int i=0;i<L->m;i++) L->x[xi(L,i,j,k)]=0;
}

/* region::setup_test (region.cc:1812-1826), one rank (ai=aj=ak=0, rank 0). */
void orc_setup_test(orc *h,int ca,int xfield,int l) {
	olev *L=&h->L[l];
	for(int k=0;k<L->o;k++) for(int j=0;j<L->n;j++) for(int i=0;i<L->m;i++) {
		double *p=xfield?&L->x[xi(L,i,j,k)]:&L->r[pi(L,i,j,k)];
		switch(ca) {
			case 0: *p=i;break;
			case 1: *p=j;break;
			case 2: *p=k;break;
			case 3: *p=k+j+i;break;
			case 4: *p=0;break;
			case 5: *p=i==7&&j==7&&k==7?1:0;break;
			case 6: *p=1;
		}
	}
}

int orc_guide_pred_iters(orc *h) {return h->iter/h->period;}

/* mg_guide::update (multigrid.cc:268-293). */
static void guide_update(orc *h,int extras) {
	int diter=-1+h->period*extras;
	if(h->use_avg) {
		double di=h->iter-h->iter_avg;
		int zscore=(int)(di/sqrt(h->iter_var));
		if(zscore>0) diter-=zscore;
		h->iter_avg=(1-h->alpha)*h->iter_avg+h->alpha*h->iter;
		h->iter_var=(1-h->alpha)*(h->iter_var+h->alpha*di*di);
	}
	h->iter+=diter;
	if(h->iter<h->period) h->iter=2*h->period-1;
}

/* multigrid::solve_v_cycles (multigrid.hh:182-219) with
 * mg_guide::set_tol (multigrid.hh:88-96) applied on the first call. */
int orc_solve_v_cycles(orc *h,double p_scale,double *res,long *sweeps) {
	long g0=h->gs_num;
	if(!h->tol_set) {
		double eps=DBL_EPSILON;
		h->tol=p_scale*p_scale*eps*eps*10000;
		h->tol_set=1;
	}
	double tol=h->tol*h->L[0].m;
	tol*=h->L[0].n;tol*=h->L[0].o;
	for(int i=0;i<orc_guide_pred_iters(h);i++) orc_v_cycle(h,0);
	int extra_rounds=0,n=0;
	while((*res=orc_l2_error_all(h,0))>tol&&n<100) {
		if(isnan(*res)) {*sweeps=h->gs_num-g0;return 2;}
		extra_rounds++;
		for(int i=0;i<extra_rounds;i++,n++) orc_v_cycle(h,0);
	}
	if(n>100) {*sweeps=h->gs_num-g0;return 1;}
	for(int i=0;i<2;i++) orc_v_cycle(h,0);
	guide_update(h,extra_rounds*(extra_rounds+1)/2);
	*sweeps=h->gs_num-g0;
	return 0;
}
