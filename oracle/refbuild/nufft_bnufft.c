/* The drop-in adapter: the reference's nufft_create2() interface
 * (src/noncart/nufft.h:48-57) implemented on libbnufft's C ABI, as a linop
 * whose lop_fun_t callbacks (src/linops/linop.h:15) forward to the library.
 * Written for this project against the reference's public headers; it is
 * the binding INTEGRATION.md describes.
 *
 * oracle/refbuild/Makefile compiles the reference's own `nufft` and `pics`
 * tools with -Dnufft_create2=nufft_create2_bnufft at their call sites
 * (src/nufft.c:226-295, src/sense/modelnc.c:52-55) and links this file and
 * libbnufft.so into them (nufft_bnufft, pics_bnufft): the reference's host
 * code, its CG included, then runs on the library's GPU NUFFT unchanged.
 * Those binaries are test infrastructure (tests/test_gpu_dropin.py).
 *
 * The reference's pointers are host memory here (its CPU build); the
 * library stages them through device buffers per call. Errors keep the
 * reference's abort semantics at the boundary (error(),
 * src/misc/misc.c:95); the library itself only returns status codes.
 */
#include <complex.h>
#include <stdbool.h>

#include "misc/types.h"
#include "misc/misc.h"
#include "misc/debug.h"
#include "linops/linop.h"
#include "noncart/nufft.h"

#include "bnufft.h"

struct bnufft_linop_s {

	linop_data_t super;
	bnufft_plan_t plan;
};

static DEF_TYPEID(bnufft_linop_s);

static void bn_check(int status)
{
	if (BNUFFT_OK != status)
		error("bnufft: %s\n", bnufft_last_error());
}

static void bn_forward(const linop_data_t* _data, complex float* dst, const complex float* src)
{
	const auto data = CAST_DOWN(bnufft_linop_s, _data);
	bn_check(bnufft_apply_forward(data->plan, dst, src, NULL));
}

static void bn_adjoint(const linop_data_t* _data, complex float* dst, const complex float* src)
{
	const auto data = CAST_DOWN(bnufft_linop_s, _data);
	bn_check(bnufft_apply_adjoint(data->plan, dst, src, NULL));
}

static void bn_normal(const linop_data_t* _data, complex float* dst, const complex float* src)
{
	const auto data = CAST_DOWN(bnufft_linop_s, _data);
	bn_check(bnufft_apply_normal(data->plan, dst, src, NULL));
}

static void bn_free(const linop_data_t* _data)
{
	const auto data = CAST_DOWN(bnufft_linop_s, _data);
	bnufft_free(data->plan);
	xfree(data);
}

struct linop_s* nufft_create2_bnufft(int N, const long ksp_dims[N], const long cim_dims[N],
		const long traj_dims[N], const complex float* traj,
		const long wgh_dims[N], const complex float* weights,
		const long bas_dims[N], const complex float* basis,
		struct nufft_conf_s conf)
{
	struct bnufft_conf bc;
	bnufft_conf_defaults(&bc);
	bc.toeplitz = conf.toeplitz;
	bc.periodic = conf.periodic;
	bc.lowmem = conf.lowmem;
	bc.os = conf.os;
	bc.width = conf.width;

	PTR_ALLOC(struct bnufft_linop_s, data);
	SET_TYPEID(bnufft_linop_s, data);

	bn_check(bnufft_create2(&data->plan, N, ksp_dims, cim_dims, traj_dims, traj,
			weights ? wgh_dims : NULL, weights, basis ? bas_dims : NULL, basis, &bc, NULL));

	debug_printf(DP_DEBUG1, "NUFFT: libbnufft (GPU)%s\n", conf.toeplitz ? ", Toeplitz" : "");

	// the k-space the linop maps to: with a basis it has the basis' frames
	// and no coefficient dim (out_dims, src/noncart/nufft.c:1018-1022, 1260)
	long out_dims[N];

	for (int i = 0; i < N; i++)
		out_dims[i] = ksp_dims[i];

	if (basis) {

		out_dims[5] = bas_dims[5];
		out_dims[6] = 1;
	}

	return linop_create(N, out_dims, N, cim_dims, CAST_UP(PTR_PASS(data)),
			bn_forward, bn_adjoint, conf.toeplitz ? bn_normal : NULL, NULL, bn_free);
}
