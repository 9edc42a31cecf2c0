/* bespirit: ESPIRiT calibration of coil sensitivities (bart ecalib) on the
 * GPU, C ABI. Part of libbnufft; statuses and bnufft_last_error() as in
 * bnufft.h.
 *
 * Replaces the reference's calibration entry points (mrirecon/bart
 * v1.0.00): extract_calib (src/misc/mri2.c:220-225) followed by calib
 * (src/calib/calib.c:797-800, declared in src/calib/calib.h), as main_ecalib
 * calls them (src/ecalib.c:150-253): bnufft_ecalib does both,
 * bnufft_calib the second alone.
 */
#ifndef BESPIRIT_H
#define BESPIRIT_H

#include "bnufft.h"

#ifdef __cplusplus
extern "C" {
#endif

/* struct ecalib_conf (src/calib/calib.h) with the options of main_ecalib
 * (src/ecalib.c:64-97). Defaults as ecalib_defaults
 * (src/calib/calib.c:693-714) and main_ecalib: kdims 6x6x6 (-k), calsize
 * 24x24x24 (-r), maps 2 (-m), threshold 0.001 (-t), numsv -1 (-n),
 * percentsv -1 (-p), crop 0.8 (-c), softcrop 0 (-S), rotphase 1 (-P clears
 * it), intensity 0 (-I), orthiter 1 with num_orthiter 30. The remaining
 * switches (weighting -W, automatic -a / a negative crop (SURE),
 * phase_normalize -N, nystroem -A, orthiter 0) are not built: a call that
 * sets one returns BNUFFT_ERR_UNSUPPORTED. */
struct bnufft_ecalib_conf {

	long kdims[3];
	long calsize[3];
	int maps;
	float threshold;
	int numsv;
	float percentsv;
	float crop;
	int softcrop;
	int rotphase;
	int orthiter;
	int num_orthiter;
	int weighting;
	int intensity;
	int phase_normalize;
	int nystroem;
};

void bnufft_ecalib_defaults(struct bnufft_ecalib_conf* conf);

/* Output dimensions for k-space ksp_dims[N] (N >= 5): sens [X, Y, Z, C,
 * maps], emaps [X, Y, Z, 1, maps], where a spatial dimension is 1 if the
 * k-space (hence the kernel) has size 1 there (src/ecalib.c:210-225). */
int bnufft_ecalib_dims(const struct bnufft_ecalib_conf* conf, int N, const long ksp_dims[], long sens_dims[], long emaps_dims[]);

/* ESPIRiT maps of Cartesian k-space ksp (dims[N], N >= 5, [X, Y, Z, C] with
 * dims 4.. of size 1; C <= 32): the calibration region is the largest fully
 * sampled centred block up to calsize, moved along the readout to its
 * largest energy. sens (and emaps, if not NULL) receive the maps and their
 * eigenvalues in the layout of bnufft_ecalib_dims. svals (host, if not
 * NULL) receives the kx*ky*kz*C singular values of the calibration matrix
 * in descending order, nkernels (if not NULL) the number of kernels kept,
 * caldims (if not NULL) the calibration region's size. ksp, sens and emaps
 * may be host or device memory. The call returns when the results are
 * written. Same results as the reference's ecalib up to float rounding;
 * the maps' global sign follows the convention that the first principal
 * coil component's last entry is real and positive (the reference takes
 * that sign from its LAPACK). The calibration matrix's eigen-decomposition
 * runs in cuSOLVER (loaded on first use, one handle per device and host
 * thread kept for the life of the process: calibrations on several threads,
 * each on its own stream, run concurrently); everything else in the
 * library's own kernels. Temporaries
 * come from a stream-ordered memory pool of the calibration's own, which
 * keeps its memory between calls. */
int bnufft_ecalib(const struct bnufft_ecalib_conf* conf, int N, const long ksp_dims[], const void* ksp,
		  void* sens, void* emaps, float* svals, long* nkernels, long caldims[3], void* stream);

/* ecalib -1 (src/ecalib.c:171-190, calone src/calib/calib.c:388-415): only
 * the first part, the kernels' low-resolution covariance, written to cov
 * as [xh, yh, zh, C(C+1)/2] (xh = 2 kx, or 1 where the k-space has size 1;
 * the packed lower triangle of each pixel's C x C matrix, the pixel index
 * fastest). svals, nkernels and caldims as for bnufft_ecalib. */
int bnufft_calone(const struct bnufft_ecalib_conf* conf, int N, const long ksp_dims[], const void* ksp,
		  void* cov, float* svals, long* nkernels, long caldims[3], void* stream);

/* calib (src/calib/calib.c:797-800, src/calib/calib.h): the same from the
 * calibration region's data cal (cal_dims[N]: [cx, cy, cz, C]) the caller
 * has extracted, into sens [X, Y, Z, C, maps] and emaps [X, Y, Z, 1, maps]
 * with X, Y, Z and maps from out_dims (out_dims[3] = C; conf->maps and
 * conf->calsize are not used). svals (host, SN >= kx*ky*kz*C entries, or
 * NULL) as for bnufft_ecalib. The kernel is 1 along a dimension where the
 * calibration data have size 1. */
int bnufft_calib(const struct bnufft_ecalib_conf* conf, int N, const long out_dims[], void* sens, void* emaps,
		 int SN, float* svals, const long cal_dims[], const void* cal, void* stream);

#ifdef __cplusplus
}
#endif

#endif
