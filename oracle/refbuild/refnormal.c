/* Checker tool, written for this project, that drives the reference's own
 * library (mrirecon/bart) through its public API to expose the Toeplitz
 * normal operator and the PSF, which the reference's command-line tools do
 * not print directly. Test infrastructure only.
 *
 *   refnormal [-P] [--no-toeplitz] [-p pattern] [-B basis] traj img out [psf_out]
 *
 * out = N^H N img, with N = nufft_create2(..., conf) and conf.toeplitz set
 * (src/noncart/nufft.c:1174-1276, normal at :1740 -> toeplitz_mult :1546).
 * With --no-toeplitz the normal is the explicit adjoint(forward(img)).
 * psf_out receives nufft_get_psf() (src/noncart/nufft.c:2022-2039).
 */
#include <complex.h>
#include <stdbool.h>
#include <string.h>
#include <stdio.h>

#include "num/multind.h"
#include "num/flpmath.h"
#include "num/init.h"
#include "misc/mmio.h"
#include "misc/mri.h"
#include "misc/misc.h"
#include "linops/linop.h"
#include "noncart/nufft.h"

int main(int argc, char* argv[])
{
	bool periodic = false;
	bool toeplitz = true;
	const char* pattern_file = NULL;
	const char* basis_file = NULL;
	int a = 1;

	while ((a < argc) && ('-' == argv[a][0])) {

		if (0 == strcmp(argv[a], "-P"))
			periodic = true;
		else if (0 == strcmp(argv[a], "--no-toeplitz"))
			toeplitz = false;
		else if ((0 == strcmp(argv[a], "-p")) && (a + 1 < argc))
			pattern_file = argv[++a];
		else if ((0 == strcmp(argv[a], "-B")) && (a + 1 < argc))
			basis_file = argv[++a];
		else
			error("unknown option %s\n", argv[a]);
		a++;
	}

	if ((argc - a) < 3)
		error("usage: refnormal [-P] [--no-toeplitz] traj img out [psf]\n");

	num_init();

	long trj_dims[DIMS];
	long img_dims[DIMS];
	complex float* traj = load_cfl(argv[a + 0], DIMS, trj_dims);
	complex float* img = load_cfl(argv[a + 1], DIMS, img_dims);

	long ksp_dims[DIMS];
	md_select_dims(DIMS, PHS1_FLAG | PHS2_FLAG, ksp_dims, trj_dims);
	md_copy_dims(DIMS - 3, ksp_dims + 3, img_dims + 3);

	struct nufft_conf_s conf = nufft_conf_defaults;
	conf.toeplitz = toeplitz;
	conf.periodic = periodic;

	long pat_dims[DIMS];
	complex float* pattern = (NULL != pattern_file) ? load_cfl(pattern_file, DIMS, pat_dims) : NULL;

	long bas_dims[DIMS];
	complex float* basis = (NULL != basis_file) ? load_cfl(basis_file, DIMS, bas_dims) : NULL;

	if (NULL != basis) {	// as the nufft tool's forward (src/nufft.c:284-288)

		ksp_dims[TE_DIM] = bas_dims[TE_DIM];
		ksp_dims[COEFF_DIM] = 1;
	}

	const struct linop_s* op = nufft_create2(DIMS, ksp_dims, img_dims, trj_dims, traj, pat_dims, pattern,
			bas_dims, basis, conf);

	complex float* out = create_cfl(argv[a + 2], DIMS, img_dims);

	if (toeplitz) {

		linop_normal(op, DIMS, img_dims, out, img);

	} else {

		complex float* ksp = md_alloc(DIMS, ksp_dims, CFL_SIZE);
		linop_forward(op, DIMS, ksp_dims, ksp, DIMS, img_dims, img);
		linop_adjoint(op, DIMS, img_dims, out, DIMS, ksp_dims, ksp);
		md_free(ksp);
	}

	if (toeplitz && (NULL == basis) && ((argc - a) > 3)) {

		long psf_dims[DIMS + 1];
		int ND = nufft_get_psf_dims(op, DIMS + 1, psf_dims);
		complex float* psf = create_cfl(argv[a + 3], ND, psf_dims);
		nufft_get_psf(op, ND, psf_dims, psf);
		unmap_cfl(ND, psf_dims, psf);
	}

	linop_free(op);
	unmap_cfl(DIMS, img_dims, out);
	unmap_cfl(DIMS, img_dims, img);
	unmap_cfl(DIMS, trj_dims, traj);

	return 0;
}
