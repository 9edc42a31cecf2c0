/* CBLAS (column-major only) over Fortran BLAS, for building the reference's
 * CPU tools as a checker and CPU baseline. Test infrastructure only.
 *
 * The reference always passes CblasColMajor (src/num/blas.c:275-630), which
 * maps one-to-one onto the Fortran interface. Routines whose Fortran symbol is
 * not exported by the installed MKL are written as plain loops.
 */
#include <assert.h>
#include <complex.h>
#include <stdlib.h>

#include "cblas.h"

extern void cgemm_(const char*, const char*, const int*, const int*, const int*, const void*, const void*, const int*,
		const void*, const int*, const void*, void*, const int*);
extern void sgemm_(const char*, const char*, const int*, const int*, const int*, const float*, const float*, const int*,
		const float*, const int*, const float*, float*, const int*);
extern void sgemv_(const char*, const int*, const int*, const float*, const float*, const int*, const float*, const int*,
		const float*, float*, const int*);
extern void caxpy_(const int*, const void*, const void*, const int*, void*, const int*);
extern void saxpy_(const int*, const float*, const float*, const int*, float*, const int*);
extern void sscal_(const int*, const float*, float*, const int*);
extern float sdot_(const int*, const float*, const int*, const float*, const int*);

static char tr(enum CBLAS_TRANSPOSE t)
{
	return (CblasNoTrans == t) ? 'N' : ((CblasTrans == t) ? 'T' : 'C');
}

void cblas_cgemm(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int M, int N, int K,
		const void* alpha, const void* A, int lda, const void* B, int ldb, const void* beta, void* C, int ldc)
{
	assert(CblasColMajor == o);
	char a = tr(ta), b = tr(tb);
	cgemm_(&a, &b, &M, &N, &K, alpha, A, &lda, B, &ldb, beta, C, &ldc);
}

void cblas_sgemm(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int M, int N, int K,
		float alpha, const float* A, int lda, const float* B, int ldb, float beta, float* C, int ldc)
{
	assert(CblasColMajor == o);
	char a = tr(ta), b = tr(tb);
	sgemm_(&a, &b, &M, &N, &K, &alpha, A, &lda, B, &ldb, &beta, C, &ldc);
}

void cblas_sgemv(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE t, int M, int N, float alpha, const float* A, int lda,
		const float* x, int incx, float beta, float* y, int incy)
{
	assert(CblasColMajor == o);
	char a = tr(t);
	sgemv_(&a, &M, &N, &alpha, A, &lda, x, &incx, &beta, y, &incy);
}

void cblas_cgemv(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE t, int M, int N, const void* _alpha, const void* _A, int lda,
		const void* _x, int incx, const void* _beta, void* _y, int incy)
{
	assert(CblasColMajor == o);
	const float complex alpha = *(const float complex*)_alpha;
	const float complex beta = *(const float complex*)_beta;
	const float complex* A = _A;
	const float complex* x = _x;
	float complex* y = _y;

	int ly = (CblasNoTrans == t) ? M : N;
	int lx = (CblasNoTrans == t) ? N : M;

	float complex* acc = calloc((size_t)ly, sizeof *acc);

	if (CblasNoTrans == t) {

		for (int j = 0; j < lx; j++)
			for (int i = 0; i < ly; i++)
				acc[i] += A[i + (long)j * lda] * x[(long)j * incx];
	} else {

		for (int i = 0; i < ly; i++)
			for (int j = 0; j < lx; j++)
				acc[i] += ((CblasConjTrans == t) ? conjf(A[j + (long)i * lda]) : A[j + (long)i * lda]) * x[(long)j * incx];
	}

	for (int i = 0; i < ly; i++)
		y[(long)i * incy] = ((0.f == beta) ? 0.f : beta * y[(long)i * incy]) + alpha * acc[i];

	free(acc);
}

void cblas_cgeru(enum CBLAS_ORDER o, int M, int N, const void* _alpha, const void* _x, int incx, const void* _y, int incy, void* _A, int lda)
{
	assert(CblasColMajor == o);
	const float complex alpha = *(const float complex*)_alpha;
	const float complex* x = _x;
	const float complex* y = _y;
	float complex* A = _A;

	for (int j = 0; j < N; j++)
		for (int i = 0; i < M; i++)
			A[i + (long)j * lda] += alpha * x[(long)i * incx] * y[(long)j * incy];
}

void cblas_sger(enum CBLAS_ORDER o, int M, int N, float alpha, const float* x, int incx, const float* y, int incy, float* A, int lda)
{
	assert(CblasColMajor == o);

	for (int j = 0; j < N; j++)
		for (int i = 0; i < M; i++)
			A[i + (long)j * lda] += alpha * x[(long)i * incx] * y[(long)j * incy];
}

void cblas_caxpy(int N, const void* alpha, const void* x, int incx, void* y, int incy)
{
	caxpy_(&N, alpha, x, &incx, y, &incy);
}

void cblas_saxpy(int N, float alpha, const float* x, int incx, float* y, int incy)
{
	saxpy_(&N, &alpha, x, &incx, y, &incy);
}

void cblas_cscal(int N, const void* _alpha, void* _x, int incx)
{
	const float complex alpha = *(const float complex*)_alpha;
	float complex* x = _x;

	for (int i = 0; i < N; i++)
		x[(long)i * incx] *= alpha;
}

void cblas_sscal(int N, float alpha, float* x, int incx)
{
	sscal_(&N, &alpha, x, &incx);
}

float cblas_sdot(int N, const float* x, int incx, const float* y, int incy)
{
	return sdot_(&N, x, &incx, y, &incy);
}

void cblas_cdotu_sub(int N, const void* _x, int incx, const void* _y, int incy, void* dotu)
{
	const float complex* x = _x;
	const float complex* y = _y;
	float complex acc = 0.f;

	for (int i = 0; i < N; i++)
		acc += x[(long)i * incx] * y[(long)i * incy];

	*(float complex*)dotu = acc;
}

void cblas_csyrk(enum CBLAS_ORDER o, enum CBLAS_UPLO uplo, enum CBLAS_TRANSPOSE t, int N, int K,
		const void* _alpha, const void* _A, int lda, const void* _beta, void* _C, int ldc)
{
	assert(CblasColMajor == o);
	const float complex alpha = *(const float complex*)_alpha;
	const float complex beta = *(const float complex*)_beta;
	const float complex* A = _A;
	float complex* C = _C;

	for (int j = 0; j < N; j++) {

		int i0 = (CblasUpper == uplo) ? 0 : j;
		int i1 = (CblasUpper == uplo) ? j : N - 1;

		for (int i = i0; i <= i1; i++) {

			float complex acc = 0.f;

			for (int k = 0; k < K; k++)
				acc += (CblasNoTrans == t) ? A[i + (long)k * lda] * A[j + (long)k * lda]
							  : A[k + (long)i * lda] * A[k + (long)j * lda];

			C[i + (long)j * ldc] = ((0.f == beta) ? 0.f : beta * C[i + (long)j * ldc]) + alpha * acc;
		}
	}
}
