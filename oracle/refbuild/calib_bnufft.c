/* The ESPIRiT drop-in: the reference's calib() (src/calib/calib.c:797-800,
 * declared in src/calib/calib.h) implemented on libbnufft's bnufft_calib.
 * Written for this project against the reference's public headers; it is
 * the binding INTEGRATION.md describes.
 *
 * oracle/refbuild/Makefile compiles the reference's own `ecalib` tool with
 * -Dcalib=calib_bnufft at its call site (src/ecalib.c:247) and links this
 * file and libbnufft.so into it (ecalib_bnufft): the reference's option
 * parsing, .cfl I/O and calibration-region extraction then feed the
 * library's GPU calibration unchanged. Test infrastructure
 * (tests/test_gpu_dropin.py).
 *
 * Options the library does not build come back as an error() here, the
 * reference's abort semantics at its boundary (src/misc/misc.c:95).
 */
#include <complex.h>
#include <stdbool.h>

#include "misc/mri.h"
#include "misc/misc.h"
#include "calib/calib.h"

#include "bespirit.h"

void calib(const struct ecalib_conf* conf, const long out_dims[DIMS], complex float* out_data, complex float* eptr,
	   int SN, float svals[SN], const long calreg_dims[DIMS], const complex float* data)
{
	if (conf->perturb > 0.)
		error("bnufft: kernel perturbation is not built\n");

	struct bnufft_ecalib_conf bc;
	bnufft_ecalib_defaults(&bc);

	for (int i = 0; i < 3; i++)
		bc.kdims[i] = conf->kdims[i];

	bc.maps = (int)out_dims[MAPS_DIM];
	bc.threshold = conf->threshold;
	bc.numsv = conf->numsv;
	bc.percentsv = conf->percentsv;
	bc.crop = conf->crop;
	bc.softcrop = conf->softcrop;
	bc.rotphase = conf->rotphase;
	bc.orthiter = conf->orthiter;
	bc.num_orthiter = conf->num_orthiter;
	bc.weighting = conf->weighting;
	bc.intensity = conf->intensity;
	bc.phase_normalize = conf->phase_normalize;
	bc.nystroem = conf->nystroem;

	if (BNUFFT_OK != bnufft_calib(&bc, DIMS, out_dims, out_data, eptr, SN, svals, calreg_dims, data, NULL))
		error("bnufft: %s\n", bnufft_last_error());
}
