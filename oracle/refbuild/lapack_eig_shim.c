/* The reference's Hermitian eigen-decomposition wrappers (src/num/lapack.c:
 * lapack_eig, lapack_eig_double) over the Fortran LAPACK that the installed
 * PyTorch CPU library exports (MKL, LP64). The reference calls cheev/zheev
 * through LAPACKE in column-major order; only the divide-and-conquer
 * variants (cheevd_, zheevd_) are exported here, which return the same
 * eigenvalues (ascending) and eigenvectors up to the sign of the real
 * tridiagonal solution (the last component of each vector is real for
 * UPLO 'U'). Test infrastructure: builds the reference's ecalib as the
 * checker of the ESPIRiT oracle. */
#include <complex.h>
#include <stdio.h>
#include <stdlib.h>

extern void cheevd_(const char* jobz, const char* uplo, const int* n, float complex* a, const int* lda, float* w,
		    float complex* work, const int* lwork, float* rwork, const int* lrwork, int* iwork,
		    const int* liwork, int* info);
extern void zheevd_(const char* jobz, const char* uplo, const int* n, double complex* a, const int* lda, double* w,
		    double complex* work, const int* lwork, double* rwork, const int* lrwork, int* iwork,
		    const int* liwork, int* info);

void lapack_eig(long N, float eigenval[N], float complex matrix[N][N]);
void lapack_eig_double(long N, double eigenval[N], double complex matrix[N][N]);

void lapack_eig(long N, float eigenval[N], float complex matrix[N][N])
{
	int n = (int)N, info = 0, q = -1, liw = 0;
	float complex wq;
	float rq;
	cheevd_("V", "U", &n, &matrix[0][0], &n, eigenval, &wq, &q, &rq, &q, &liw, &q, &info);
	int lw = (int)crealf(wq), lrw = (int)rq, li = liw;
	float complex* work = malloc(sizeof(float complex) * (size_t)lw);
	float* rwork = malloc(sizeof(float) * (size_t)lrw);
	int* iwork = malloc(sizeof(int) * (size_t)li);
	cheevd_("V", "U", &n, &matrix[0][0], &n, eigenval, work, &lw, rwork, &lrw, iwork, &li, &info);
	free(work);
	free(rwork);
	free(iwork);
	if (0 != info) {
		fprintf(stderr, "LAPACK: cheev failed.\n");
		abort();
	}
}

void lapack_eig_double(long N, double eigenval[N], double complex matrix[N][N])
{
	int n = (int)N, info = 0, q = -1, liw = 0;
	double complex wq;
	double rq;
	zheevd_("V", "U", &n, &matrix[0][0], &n, eigenval, &wq, &q, &rq, &q, &liw, &q, &info);
	int lw = (int)creal(wq), lrw = (int)rq, li = liw;
	double complex* work = malloc(sizeof(double complex) * (size_t)lw);
	double* rwork = malloc(sizeof(double) * (size_t)lrw);
	int* iwork = malloc(sizeof(int) * (size_t)li);
	zheevd_("V", "U", &n, &matrix[0][0], &n, eigenval, work, &lw, rwork, &lrw, iwork, &li, &info);
	free(work);
	free(rwork);
	free(iwork);
	if (0 != info) {
		fprintf(stderr, "LAPACK: zheev failed.\n");
		abort();
	}
}
