/* Standard CBLAS prototypes for the subset the reference calls
 * (src/num/blas.c in mrirecon/bart), written for this project.
 * Implemented in cblas_shim.c over the Fortran BLAS entry points that
 * PyTorch's CPU library exports (MKL), with plain loops for the rest.
 * Test infrastructure only.
 */
#ifndef REFBUILD_CBLAS_H
#define REFBUILD_CBLAS_H

#ifdef __cplusplus
extern "C" {
#endif

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };

typedef enum CBLAS_ORDER CBLAS_LAYOUT;

void cblas_cgemm(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int M, int N, int K,
		const void* alpha, const void* A, int lda, const void* B, int ldb, const void* beta, void* C, int ldc);
void cblas_cgemv(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE t, int M, int N, const void* alpha, const void* A, int lda,
		const void* x, int incx, const void* beta, void* y, int incy);
void cblas_cgeru(enum CBLAS_ORDER o, int M, int N, const void* alpha, const void* x, int incx, const void* y, int incy, void* A, int lda);
void cblas_caxpy(int N, const void* alpha, const void* x, int incx, void* y, int incy);
void cblas_cscal(int N, const void* alpha, void* x, int incx);
void cblas_cdotu_sub(int N, const void* x, int incx, const void* y, int incy, void* dotu);
void cblas_csyrk(enum CBLAS_ORDER o, enum CBLAS_UPLO uplo, enum CBLAS_TRANSPOSE t, int N, int K,
		const void* alpha, const void* A, int lda, const void* beta, void* C, int ldc);

void cblas_sgemm(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int M, int N, int K,
		float alpha, const float* A, int lda, const float* B, int ldb, float beta, float* C, int ldc);
void cblas_sgemv(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE t, int M, int N, float alpha, const float* A, int lda,
		const float* x, int incx, float beta, float* y, int incy);
void cblas_sger(enum CBLAS_ORDER o, int M, int N, float alpha, const float* x, int incx, const float* y, int incy, float* A, int lda);
void cblas_saxpy(int N, float alpha, const float* x, int incx, float* y, int incy);
void cblas_sscal(int N, float alpha, float* x, int incx);
float cblas_sdot(int N, const float* x, int incx, const float* y, int incy);

#ifdef __cplusplus
}
#endif
#endif
