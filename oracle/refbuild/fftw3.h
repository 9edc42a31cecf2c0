/* Minimal single-precision FFTW3 API declarations, written for this project.
 *
 * Only what the reference's FFT planner uses (src/num/fft_plan.c:187-245, 279,
 * 290, 414-427 in mrirecon/bart) is declared. The implementation lives in
 * fftw_mkl_shim.c and runs the transforms through Intel MKL's DFTI interface,
 * which the installed PyTorch CPU library exports. Test infrastructure only:
 * used to build the reference's own CPU tools as a checker and CPU baseline.
 */
#ifndef REFBUILD_FFTW3_H
#define REFBUILD_FFTW3_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct refbuild_fftwf_plan_s* fftwf_plan;

typedef struct {
	ptrdiff_t n;
	ptrdiff_t is;
	ptrdiff_t os;
} fftwf_iodim64;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftwf_plan fftwf_plan_guru64_dft(int rank, const fftwf_iodim64* dims,
		int howmany_rank, const fftwf_iodim64* howmany_dims,
		fftwf_complex* in, fftwf_complex* out, int sign, unsigned flags);

void fftwf_execute_dft(const fftwf_plan p, fftwf_complex* in, fftwf_complex* out);
void fftwf_destroy_plan(fftwf_plan p);

int fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int nthreads);
void fftwf_cleanup_threads(void);
void fftwf_cleanup(void);

int fftwf_import_wisdom_from_filename(const char* filename);
int fftwf_export_wisdom_to_filename(const char* filename);

#ifdef __cplusplus
}
#endif
#endif
