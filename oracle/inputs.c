/* Seeded benchmark inputs for the oracle side (TEST INFRASTRUCTURE ONLY).
 *
 * The reference ships no variable-coefficient problem class, so the
 * benchmark's inputs come from this repository's own generator
 * (pgmg_b200/csrc/problems.cpp).  The reference arm of bench.py and the
 * CPU-baseline pools must not load the product library, so this file
 * restates that generator for the oracle library; tests/test_oracle_inputs.py
 * checks that both give the same arrays bit for bit.  Built with
 * -ffp-contract=off (no fused multiply-add, like the product's x86-64 host
 * build) and linked against the same libm.
 *
 *  * Gaussian field: cell-centred g ~ N(0,1) per cell, SplitMix64 of
 *    (seed * FNV prime) ^ counter, Box-Muller (cos branch), convolved with a
 *    separable Gaussian of width w cells truncated at ceil(4w), reflective
 *    (half-sample-symmetric) edges, then normalised to zero mean and unit
 *    variance with per-plane partial sums added in plane order.
 *  * kappa = exp(sigma * g).
 *  * Q1 trilinear FEM stencil of -div(kappa grad u), h = 1/(max(m,n,o)-1);
 *    Dirichlet boundary nodes are one-entry rows 8/3 h mean(kappa of the
 *    cells touching the node), box [0,1)^3.
 *  * RHS: interior nodes uniform[-1,1] from SplitMix64, boundary 0.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "pgmg_oracle.h"

static uint64_t sm64(uint64_t z) {
	z+=0x9E3779B97F4A7C15ull;
	z=(z^(z>>30))*0xBF58476D1CE4E5B9ull;
	z=(z^(z>>27))*0x94D049BB133111EBull;
	return z^(z>>31);
}

/* (0,1]: 53 random bits plus one unit in the last place, so log() is finite. */
static double open01(uint64_t b) {return ((b>>11)+1)*(1.0/9007199254740992.0);}

static long refl(long t,long len) {
	long per=2*len;
	if(len==1) return 0;
	t%=per;
	if(t<0) t+=per;
	return t<len?t:per-1-t;
}

/* One axis of the separable convolution, out-of-place. */
static void conv_axis(double *a,double *tmp,long nx,long ny,long nz,int axis,const double *w,int rad) {
	long len=axis==0?nx:(axis==1?ny:nz);
	long stride=axis==0?1:(axis==1?nx:nx*ny);
	long lines=nx*ny*nz/len,l;
#pragma omp parallel for schedule(static)
	for(l=0;l<lines;l++) {
		long base,t;
		if(axis==0) base=l*nx;
		else if(axis==1) base=(l/nx)*nx*ny+(l%nx);
		else base=l;
		for(t=0;t<len;t++) {
			double s=0;
			int d;
			for(d=-rad;d<=rad;d++) s+=w[d+rad]*a[base+refl(t+d,len)*stride];
			tmp[base+t*stride]=s;
		}
	}
	memcpy(a,tmp,sizeof(double)*nx*ny*nz);
}

int orc_input_gauss(int m,int n,int o,uint64_t seed,double width,double *out) {
	long nx=m-1,ny=n-1,nz=o-1,nc,c,k;
	double *g,*ps,*pq,mean=0,var=0,inv_sd;
	if(m<2||n<2||o<2||!out) return 1;
	nc=nx*ny*nz;
	g=(double*)malloc(sizeof(double)*nc);
	if(!g) return 1;
#pragma omp parallel for schedule(static)
	for(c=0;c<nc;c++) {
		uint64_t key=seed*0x100000001B3ull;
		double u1=open01(sm64(key^(2*(uint64_t)c))),u2=open01(sm64(key^(2*(uint64_t)c+1)));
		g[c]=sqrt(-2.0*log(u1))*cos(6.283185307179586*u2);
	}
	if(width>0) {
		int rad=(int)ceil(4*width),d;
		double *w=(double*)malloc(sizeof(double)*(2*rad+1)),ws=0,*tmp;
		tmp=(double*)malloc(sizeof(double)*nc);
		if(!w||!tmp) {free(g);free(w);free(tmp);return 1;}
		for(d=-rad;d<=rad;d++) ws+=(w[d+rad]=exp(-0.5*d*d/(width*width)));
		for(d=0;d<2*rad+1;d++) w[d]/=ws;
		conv_axis(g,tmp,nx,ny,nz,0,w,rad);
		conv_axis(g,tmp,nx,ny,nz,1,w,rad);
		conv_axis(g,tmp,nx,ny,nz,2,w,rad);
		free(w);free(tmp);
	}
	ps=(double*)malloc(sizeof(double)*nz);
	pq=(double*)malloc(sizeof(double)*nz);
	if(!ps||!pq) {free(g);free(ps);free(pq);return 1;}
#pragma omp parallel for schedule(static)
	for(k=0;k<nz;k++) {
		double s=0;
		long q;
		for(q=k*nx*ny;q<(k+1)*nx*ny;q++) s+=g[q];
		ps[k]=s;
	}
	for(k=0;k<nz;k++) mean+=ps[k];
	mean/=(double)nc;
#pragma omp parallel for schedule(static)
	for(k=0;k<nz;k++) {
		double s=0;
		long q;
		for(q=k*nx*ny;q<(k+1)*nx*ny;q++) s+=(g[q]-mean)*(g[q]-mean);
		pq[k]=s;
	}
	for(k=0;k<nz;k++) var+=pq[k];
	var/=(double)nc;
	inv_sd=var>0?1.0/sqrt(var):0.0;
#pragma omp parallel for schedule(static)
	for(c=0;c<nc;c++) out[c]=(g[c]-mean)*inv_sd;
	free(g);free(ps);free(pq);
	return 0;
}

int orc_input_kappa(int m,int n,int o,double sigma,uint64_t seed,double width,double *kappa) {
	long nc=(long)(m-1)*(n-1)*(o-1),c;
	if(orc_input_gauss(m,n,o,seed,width,kappa)) return 1;
#pragma omp parallel for schedule(static)
	for(c=0;c<nc;c++) kappa[c]=exp(sigma*kappa[c]);
	return 0;
}

int orc_input_q1(int m,int n,int o,const double *kappa,double *c27,int *S6) {
	const long nx=m-1,ny=n-1;
	const int mx=m>n?(m>o?m:o):(n>o?n:o);
	const double h=1.0/(double)(mx-1);
	const double khat[4]={1.0/3.0,0.0,-1.0/12.0,-1.0/12.0};
	long k;
	if(m<2||n<2||o<2||!c27) return 1;
#pragma omp parallel for schedule(static)
	for(k=0;k<o;k++) {
		long j,i;
		for(j=0;j<n;j++) for(i=0;i<m;i++) {
			long p=i+(long)m*(j+(long)n*k);
			double *c=c27+27*p;
			int q,in=i>0&&i<m-1&&j>0&&j<n-1&&k>0&&k<o-1;
			for(q=0;q<27;q++) c[q]=0;
			if(in) {
				int ce,cb,ca,ee,bb,aa;
				for(ce=-1;ce<=0;ce++) for(cb=-1;cb<=0;cb++) for(ca=-1;ca<=0;ca++) {
					double ke=h*(kappa?kappa[(i+ca)+nx*((j+cb)+ny*(k+ce))]:1.0);
					for(ee=0;ee<2;ee++) for(bb=0;bb<2;bb++) for(aa=0;aa<2;aa++) {
						int diff=(aa!=-ca)+(bb!=-cb)+(ee!=-ce);
						c[(aa+ca+1)+3*(bb+cb+1)+9*(ee+ce+1)]+=ke*khat[diff];
					}
				}
			} else {
				double s=0;
				int cnt=0,e,b,a;
				for(e=-1;e<=0;e++) for(b=-1;b<=0;b++) for(a=-1;a<=0;a++) {
					long ci=i+a,cj=j+b,ck=k+e;
					if(ci<0||cj<0||ck<0||ci>=nx||cj>=ny||ck>=o-1) continue;
					s+=kappa?kappa[ci+nx*(cj+ny*ck)]:1.0;
					cnt++;
				}
				c[13]=8.0/3.0*h*(s/cnt);
			}
			if(S6) {
				int *s=S6+6*p;
				s[0]=s[2]=s[4]=in?-1:0;
				s[1]=s[3]=s[5]=in?2:1;
			}
		}
	}
	return 0;
}

int orc_input_rhs(int m,int n,int o,uint64_t seed,double *r) {
	uint64_t key=(seed+0x5851F42D4C957F2Dull)*0x2545F4914F6CDD1Dull;
	long k;
	if(m<1||n<1||o<1||!r) return 1;
#pragma omp parallel for schedule(static)
	for(k=0;k<o;k++) {
		long j,i;
		for(j=0;j<n;j++) for(i=0;i<m;i++) {
			long p=i+(long)m*(j+(long)n*k);
			int in=i>0&&i<m-1&&j>0&&j<n-1&&k>0&&k<o-1;
			r[p]=in?2.0*(open01(sm64(key^(uint64_t)p))-0.5):0.0;
		}
	}
	return 0;
}
