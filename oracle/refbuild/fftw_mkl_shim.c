/* FFTW3 guru64 single-precision complex DFT implemented over Intel MKL DFTI.
 *
 * Test infrastructure only. The reference (mrirecon/bart) links FFTW3f for its
 * CPU FFTs (src/num/fft_plan.c:187-245); FFTW is not installed on these
 * machines, but PyTorch's CPU library exports MKL's DFTI entry points, so the
 * reference's CPU tools are built against this translation layer instead.
 *
 * Semantics kept from FFTW: sign -1 is the forward transform e^{-2 pi i jk/n},
 * no normalisation, arbitrary element strides for the transform and
 * "howmany" (batch) dimensions, in-place when in == out.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <complex.h>

#include "fftw3.h"

/* MKL DFTI public ABI (documented configuration parameter and value codes). */
typedef void* DFTI_DESCRIPTOR_HANDLE;
typedef long MKL_LONG;

enum { DFTI_PRECISION_ = 3, DFTI_FORWARD_SCALE_ = 4, DFTI_BACKWARD_SCALE_ = 5,
	DFTI_NUMBER_OF_TRANSFORMS_ = 7, DFTI_PLACEMENT_ = 11,
	DFTI_INPUT_STRIDES_ = 12, DFTI_OUTPUT_STRIDES_ = 13,
	DFTI_INPUT_DISTANCE_ = 14, DFTI_OUTPUT_DISTANCE_ = 15 };

enum { DFTI_COMPLEX_ = 32, DFTI_SINGLE_ = 35, DFTI_INPLACE_ = 43, DFTI_NOT_INPLACE_ = 44 };

extern MKL_LONG DftiCreateDescriptor_s_md(DFTI_DESCRIPTOR_HANDLE*, int domain, MKL_LONG dim, MKL_LONG* sizes);
extern MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE, int param, ...);
extern MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE);
extern MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE, void*, ...);
extern MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE, void*, ...);
extern MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE*);
extern char* DftiErrorMessage(MKL_LONG);

enum { MAXD = 16 };

struct refbuild_fftwf_plan_s {

	int rank;
	fftwf_iodim64 dims[MAXD];
	int loop_rank;			/* batch dims looped in C (all but the batched one) */
	fftwf_iodim64 loops[MAXD];
	int sign;
	int inplace;
	int trivial;			/* rank 0: plain strided copy */
	fftwf_iodim64 batch;		/* batch dim handed to MKL as NUMBER_OF_TRANSFORMS */
	DFTI_DESCRIPTOR_HANDLE desc;
};

static void check(MKL_LONG st, const char* what)
{
	if (0 != st) {

		fprintf(stderr, "fftw-mkl shim: %s failed: %s\n", what, DftiErrorMessage(st));
		abort();
	}
}

fftwf_plan fftwf_plan_guru64_dft(int rank, const fftwf_iodim64* dims,
		int howmany_rank, const fftwf_iodim64* howmany_dims,
		fftwf_complex* in, fftwf_complex* out, int sign, unsigned flags)
{
	(void)flags;

	if (rank > MAXD || howmany_rank > MAXD)
		return NULL;

	struct refbuild_fftwf_plan_s* p = calloc(1, sizeof *p);

	p->sign = sign;
	p->inplace = ((void*)in == (void*)out);

	/* drop singleton transform dims (MKL rejects none, but keeps it simple) */
	p->rank = 0;

	for (int i = 0; i < rank; i++)
		if (dims[i].n > 1)
			p->dims[p->rank++] = dims[i];

	/* choose the largest batch dim for MKL's NUMBER_OF_TRANSFORMS */
	int bi = -1;

	for (int i = 0; i < howmany_rank; i++)
		if ((howmany_dims[i].n > 1) && ((-1 == bi) || (howmany_dims[i].n > howmany_dims[bi].n)))
			bi = i;

	p->batch = (-1 == bi) ? (fftwf_iodim64){ 1, 0, 0 } : howmany_dims[bi];
	p->loop_rank = 0;

	for (int i = 0; i < howmany_rank; i++)
		if ((i != bi) && (howmany_dims[i].n > 1))
			p->loops[p->loop_rank++] = howmany_dims[i];

	if (0 == p->rank) {

		p->trivial = 1;
		return p;
	}

	MKL_LONG lengths[MAXD];
	MKL_LONG istr[MAXD + 1];
	MKL_LONG ostr[MAXD + 1];

	istr[0] = 0;
	ostr[0] = 0;

	for (int i = 0; i < p->rank; i++) {

		lengths[i] = p->dims[i].n;
		istr[i + 1] = p->dims[i].is;
		ostr[i + 1] = p->dims[i].os;
	}

	check(DftiCreateDescriptor_s_md(&p->desc, DFTI_COMPLEX_, p->rank, lengths), "create");
	check(DftiSetValue(p->desc, DFTI_PLACEMENT_, p->inplace ? DFTI_INPLACE_ : DFTI_NOT_INPLACE_), "placement");
	check(DftiSetValue(p->desc, DFTI_INPUT_STRIDES_, istr), "input strides");
	check(DftiSetValue(p->desc, DFTI_OUTPUT_STRIDES_, ostr), "output strides");

	if (p->batch.n > 1) {

		check(DftiSetValue(p->desc, DFTI_NUMBER_OF_TRANSFORMS_, (MKL_LONG)p->batch.n), "transforms");
		check(DftiSetValue(p->desc, DFTI_INPUT_DISTANCE_, (MKL_LONG)p->batch.is), "input distance");
		check(DftiSetValue(p->desc, DFTI_OUTPUT_DISTANCE_, (MKL_LONG)p->batch.os), "output distance");
	}

	check(DftiCommitDescriptor(p->desc), "commit");

	return p;
}

static void exec_loop(const struct refbuild_fftwf_plan_s* p, int l, float complex* in, float complex* out)
{
	if (l == p->loop_rank) {

		if (p->trivial) {

			/* rank-0 transform: strided copy over the batch dim */
			for (ptrdiff_t b = 0; b < p->batch.n; b++)
				out[b * p->batch.os] = in[b * p->batch.is];

			return;
		}

		if (p->inplace)
			check((-1 == p->sign) ? DftiComputeForward(p->desc, (void*)in) : DftiComputeBackward(p->desc, (void*)in), "compute");
		else
			check((-1 == p->sign) ? DftiComputeForward(p->desc, (void*)in, (void*)out) : DftiComputeBackward(p->desc, (void*)in, (void*)out), "compute");

		return;
	}

	for (ptrdiff_t j = 0; j < p->loops[l].n; j++)
		exec_loop(p, l + 1, in + j * p->loops[l].is, out + j * p->loops[l].os);
}

void fftwf_execute_dft(const fftwf_plan p, fftwf_complex* in, fftwf_complex* out)
{
	exec_loop(p, 0, (float complex*)in, (float complex*)out);
}

void fftwf_destroy_plan(fftwf_plan p)
{
	if (NULL == p)
		return;

	if (!p->trivial)
		DftiFreeDescriptor(&p->desc);

	free(p);
}

int fftwf_init_threads(void) { return 1; }
void fftwf_plan_with_nthreads(int nthreads) { (void)nthreads; }
void fftwf_cleanup_threads(void) { }
void fftwf_cleanup(void) { }
int fftwf_import_wisdom_from_filename(const char* filename) { (void)filename; return 0; }
int fftwf_export_wisdom_to_filename(const char* filename) { (void)filename; return 0; }
