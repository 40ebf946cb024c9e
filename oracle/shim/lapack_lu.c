/* Stand-in for the two LAPACK routines the PGMG reference calls on its
 * coarsest level (region_tr.cc:11-15, used at region_tr.cc:519 and :552).
 *
 * TEST INFRASTRUCTURE ONLY (oracle).  No system LAPACK exists in this image,
 * and the reference pins no LAPACK version (config/config.mk.linux:11 links
 * plain -llapack -lblas), so this file restates the published algorithms:
 *   dgetrf_: LU factorisation with partial (row) pivoting, column-major,
 *            the unblocked right-looking form of LAPACK's DGETF2 (Golub & Van
 *            Loan, Matrix Computations, Alg. 3.4.1): for each column j pick the
 *            first row of largest |a_ij| (i >= j), swap it into row j across
 *            the whole matrix, scale the sub-column by 1/a_jj and apply the
 *            rank-1 update to the trailing block.  info = index (1-based) of
 *            the first exactly-zero pivot, 0 otherwise; factorisation carries
 *            on past a zero pivot as LAPACK does.
 *   dgetrs_: trans='N' solve: apply the recorded row interchanges to b in
 *            order (DLASWP), forward substitution with the unit lower factor,
 *            back substitution with the upper factor.
 * The tests check this restatement against scipy's LAPACK dgetrf/dgetrs.
 */
#include <math.h>

int dgetrf_(int *m_,int *n_,double *a,int *lda_,int *ipiv,int *info) {
	int m=*m_,n=*n_,lda=*lda_,mn=m<n?m:n,i,j,k,p;
	*info=0;
	for(j=0;j<mn;j++) {
		/* Pivot search: first index of the maximum absolute value. */
		p=j;
		double best=fabs(a[j+j*lda]);
		for(i=j+1;i<m;i++) {
			double v=fabs(a[i+j*lda]);
			if(v>best) {best=v;p=i;}
		}
		ipiv[j]=p+1;
		if(a[p+j*lda]!=0.0) {
			if(p!=j) for(k=0;k<n;k++) {
				double t=a[j+k*lda];a[j+k*lda]=a[p+k*lda];a[p+k*lda]=t;
			}
			double r=1.0/a[j+j*lda];
			for(i=j+1;i<m;i++) a[i+j*lda]*=r;
		} else if(*info==0) *info=j+1;
		/* Rank-1 update of the trailing block. */
		for(k=j+1;k<n;k++) {
			double u=a[j+k*lda];
			if(u!=0.0) for(i=j+1;i<m;i++) a[i+k*lda]-=a[i+j*lda]*u;
		}
	}
	return 0;
}

int dgetrs_(char *trans,int *n_,int *nrhs_,double *a,int *lda_,int *ipiv,double *b,int *ldb_,int *info) {
	int n=*n_,nrhs=*nrhs_,lda=*lda_,ldb=*ldb_,i,j,c;
	*info=0;
	if(*trans!='N'&&*trans!='n') {*info=-1;return 0;}
	for(c=0;c<nrhs;c++) {
		double *x=b+c*ldb;
		for(i=0;i<n;i++) {
			int p=ipiv[i]-1;
			if(p!=i) {double t=x[i];x[i]=x[p];x[p]=t;}
		}
		/* L y = P b, unit diagonal, column-oriented as DTRSM does. */
		for(j=0;j<n;j++) {
			double xj=x[j];
			if(xj!=0.0) for(i=j+1;i<n;i++) x[i]-=xj*a[i+j*lda];
		}
		/* U x = y, column-oriented back substitution. */
		for(j=n-1;j>=0;j--) {
			if(x[j]!=0.0) {
				x[j]/=a[j+j*lda];
				double xj=x[j];
				for(i=0;i<j;i++) x[i]-=xj*a[i+j*lda];
			}
		}
	}
	return 0;
}
