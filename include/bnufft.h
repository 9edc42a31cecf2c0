/* bnufft: B200-native NUFFT and CG-SENSE, C ABI.
 *
 * Drop-in boundary for the NUFFT linop and the CG-SENSE solve of
 * mrirecon/bart v1.0.00. Every entry point takes plain pointers and sizes and
 * returns a status code (0 = success); on failure bnufft_last_error() gives
 * a message. Arrays are BART arrays: column-major complex float with N (16)
 * dimensions in the reference's order (src/misc/mri.h:12-35). Data pointers
 * may be host or device memory (decided per call from the pointer, as the
 * reference does with cuda_ondevice(), src/num/gpuops.c:445); host data is
 * staged through device buffers. "stream" is a cudaStream_t (NULL: default
 * stream). There is no CPU fallback: without a usable CUDA device every
 * call fails with BNUFFT_ERR_CUDA.
 * The library keeps per-device tables (FFT twiddles, the allocation-free
 * entry point's scratch contents) for the life of the process: a
 * cudaDeviceReset() while it is loaded destroys them without its knowledge
 * and is not supported.
 */
#ifndef BNUFFT_H
#define BNUFFT_H

#ifdef __cplusplus
extern "C" {
#endif

enum bnufft_status {
	BNUFFT_OK = 0,
	BNUFFT_ERR_ARG = 1,		/* bad dimensions / options */
	BNUFFT_ERR_UNSUPPORTED = 2,	/* valid for the reference, not built here */
	BNUFFT_ERR_CUDA = 3,		/* CUDA runtime error (message has details) */
	BNUFFT_ERR_NOMEM = 4,
};

/* NUFFT configuration: the subset of struct nufft_conf_s
 * (src/noncart/nufft.h:7-30) this build implements. Defaults as
 * nufft_conf_defaults (src/noncart/nufft.c:53-74): toeplitz 1, periodic 0,
 * os 2, width 6. deterministic selects fixed-order (atomic-free) gridding. */
struct bnufft_conf {

	int toeplitz;
	int periodic;
	int deterministic;
	float os;		/* 2, or in (1, 4] with an even lround(os N): the
				   reference's chained NUFFT (src/noncart/nufft_chain.c),
				   which has no Toeplitz normal (toeplitz is then ignored;
				   the normal is adjoint(forward)) */
	float width;
	int bin;		/* gridding bin edge in grid cells (a power of two 8..128);
				   0 = default (32 in 2D, 16 in 3D). A tuning knob with no
				   effect on results (bnufft_autotune_bins picks it). */
	int lowmem;		/* --lowmem (nufft_conf_s.lowmem): the apply calls hold
				   the oversampled grid of one coil at a time (same
				   results, coil passes one after another); not with
				   per-coil weights */
};

typedef struct bnufft_plan_s* bnufft_plan_t;

/* Defaults as nufft_conf_defaults. */
void bnufft_conf_defaults(struct bnufft_conf* conf);

/* Replaces nufft_create2() (src/noncart/nufft.h:48-57, src/noncart/nufft.c:1174).
 * ksp_dims [1, Mr, Ms, C, ...], cim_dims [X, Y, Z, C, ...], traj_dims
 * [3, Mr, Ms, 1, ...], traj complex float (real parts used). weights
 * (density weights or the -p sampling pattern, nufft_set_traj
 * src/noncart/nufft.c:1041-1049) may be NULL, [1, Mr, Ms] or match the
 * k-space dims (per coil; not with the Toeplitz PSF or --lowmem): the
 * forward multiplies its k-space by them, the adjoint its input by their
 * conjugate (src/noncart/nufft.c:1457, 1477).
 * basis (bart nufft/pics -B, the subspace basis of nufft_set_traj,
 * src/noncart/nufft.c:1018-1042) may be NULL or [1, 1, 1, 1, 1, T, K]
 * with K <= 32: then cim_dims has the K coefficients in dim 6 (dim 5 = 1),
 * ksp_dims the T frames in dim 5 (dim 6 = 1), traj_dims 1 or T frames in
 * dim 5, and weights are [1, Mr, Ms, 1, 1, T or 1]. The forward is
 * y_t = sum_k B[t, k] NUFFT_t(x_k) (:1443-1453), the normal with Toeplitz
 * the block PSF P[k, k'] = sum_t conj(B[t, k]) B[t, k'] PSF_t (:470-505,
 * 1546-1625). Not with --lowmem, trajectory updates, nufft -i or
 * bnufft_get_psf. The plan copies
 * the trajectory and weights (the caller keeps its buffers) and, with
 * conf->toeplitz, computes the PSF on the device (compute_psf2,
 * src/noncart/nufft.c:727-776). */
int bnufft_create2(bnufft_plan_t* plan, int N, const long ksp_dims[], const long cim_dims[],
		const long traj_dims[], const void* traj,
		const long wgh_dims[], const void* weights,
		const long bas_dims[], const void* basis,
		const struct bnufft_conf* conf, void* stream);

/* Linop callbacks of the NUFFT (lop_fun_t, src/linops/linop.c:300):
 * forward  = nufft_apply_forward (src/noncart/nufft.c:1388), cim -> ksp
 * adjoint  = nufft_apply_adjoint (src/noncart/nufft.c:1462), ksp -> cim
 * normal   = nufft_apply_normal (src/noncart/nufft.c:1740), cim -> cim;
 *            Toeplitz embedding when the plan has a PSF, else adjoint(forward). */
int bnufft_apply_forward(bnufft_plan_t plan, void* dst, const void* src, void* stream);
int bnufft_apply_adjoint(bnufft_plan_t plan, void* dst, const void* src, void* stream);
int bnufft_apply_normal(bnufft_plan_t plan, void* dst, const void* src, void* stream);

/* Replaces nufft_get_psf_dims / nufft_get_psf (src/noncart/nufft.c:2008-2039):
 * the PSF in the reference's decomposed layout [X, Y, Z, 1, ..., 2^d] with
 * N+1 dims. psf_dims receives N+1 entries. */
int bnufft_get_psf_dims(bnufft_plan_t plan, int ND, long psf_dims[]);
int bnufft_get_psf(bnufft_plan_t plan, int ND, const long psf_dims[], void* psf, void* stream);

/* Replaces nufft_update_traj (src/noncart/nufft.c:2041-2054) for a
 * trajectory of unchanged dims. The plan keeps its weights, as the
 * reference does when its weights argument is NULL; the sample bins (and
 * the CSR of the deterministic mode) and, with Toeplitz, the PSF are
 * rebuilt for the new trajectory, so the plan then equals one created with
 * it. */
int bnufft_update_traj(bnufft_plan_t plan, int N, const long traj_dims[], const void* traj, void* stream);

/* bart nufft -i [-c] -l lambda -m maxiter (src/nufft.c:250-263): CG
 * (conjgrad, src/iter/italgos.c:497) over all coil images jointly on
 * (N^H N + lambda) x = N^H y, through lsqr2_create (src/iter/lsqr.c:78-167);
 * with precond the reference's circulant preconditioner
 * (nufft_precond_create, src/noncart/precond.c:95) is chained in front of
 * the normal operator and the right-hand side. img: cim dims; ksp: ksp dims. */
int bnufft_nufft_inverse(bnufft_plan_t plan, void* img, const void* ksp, float lambda, int maxiter,
		int precond, void* stream);

/* linop_free() of a NUFFT linop (nufft_free_data, src/noncart/nufft.c:1334). */
void bnufft_free(bnufft_plan_t plan);

/* Forward NUFFT of one 2D image that allocates no device memory. It has no
 * counterpart in the reference. It serves callers that cannot allocate
 * while they run: a scanner's real-time reconstruction process that reserves
 * its device memory up front, or code that must not pay cudaMalloc's implicit
 * device-wide synchronisation (or risk its failure) mid-stream. Results equal
 * bnufft_apply_forward of a plan with default options (os 2, width 6,
 * non-periodic).
 * traj: device [3, M] complex float; img: device [X, Y] complex float;
 * ksp: device [M] complex float. Limits: X, Y powers of two from 8 to 256,
 * M <= 262144; larger requests return BNUFFT_ERR_ARG.
 * Scratch: one file-scope device array of about 7.4 MB, held by every GPU
 * that loads the library until exit and shared by all calls, so calls that
 * overlap on the GPU race and must be serialised by the caller. The first
 * call on a device sets up the array's tables and synchronises `stream`
 * once; make that first call before any stream capture. */
int bnufft_forward2d_noalloc(long X, long Y, long M, const void* traj, const void* img, void* ksp, void* stream);

/* --- CG-SENSE: bart pics -l2 -r lambda -i iter -t traj ksp sens out ------- */

struct bnufft_pics_conf {

	float lambda;		/* -r (l2 regularisation), src/grecon/optreg.c:382-393 */
	int maxiter;		/* -i, default 30 (src/pics.c:82) */
	float tol;		/* CG stop: ||r|| <= tol * ||A^H y|| (iter_conjgrad_defaults.tol = 0) */
	float scaling;		/* -w: 0 = estimate (src/pics.c:499-530) */
	int rescale;		/* -S */
	int toeplitz;		/* default 1 (src/pics.c:90-91); 0 = --no-toeplitz */
	int periodic;
	int deterministic;
	int bin;		/* gridding bin edge of the NUFFT (bnufft_conf.bin) */
	int precond;		/* 0: plain CG (the reference's pics); 1: flexible CG with
				   the circulant preconditioner of the NUFFT's PSF
				   (nufft_precond_create, src/noncart/precond.c:48-164);
				   2: flexible CG with the padded-circulant preconditioner
				   (as 3) plus the learned correction
				   (bnufft_pics_set_precnet);
				   3: flexible CG with the padded-circulant preconditioner
				   (no counterpart in the reference): the Toeplitz
				   operator's own 2N (or embedding) circulant inverted,
				   crop F^-1 (|P| + mu)^-1 F pad, mu from lambda.
				   1, 2 and 3 need the Toeplitz normal operator. */
	int ref_scalars;	/* plain CG (precond 0) keeps ||r||^2, p^H A p, alpha and
				   beta in float32 as conjgrad stores them
				   (src/iter/italgos.c:518-554), so unconverged iterates
				   follow the reference's; 0 = float64 scalars. Default 1. */
	int net_iters;		/* precond 2: the learned correction is used in the first
				   net_iters iterations only (0 = until the stall test
				   switches it off). With a budget flexible CG keeps
				   one direction (short recurrence). Default 1. */
};

typedef struct bnufft_pics_s* bnufft_pics_t;

void bnufft_pics_conf_defaults(struct bnufft_pics_conf* conf);

/* Builds the SENSE model A = NUFFT o maps (sense_nc_init,
 * src/sense/modelnc.c:28-67; maps2_create src/sense/model.c:93) for
 * ksp_dims [1, Mr, Ms, C], sens_dims [X, Y, Z, C], traj_dims [3, Mr, Ms].
 * Host arrays are copied on the library's per-thread copy stream; the call
 * returns once they have been read (the caller may reuse them), while the
 * model's set-up kernels may still run on the stream. */
int bnufft_pics_create(bnufft_pics_t* pics, int N, const long ksp_dims[], const long sens_dims[],
		const long traj_dims[], const void* traj, const void* sens,
		const struct bnufft_pics_conf* conf, void* stream);

/* One reconstruction (main_pics CG branch, src/pics.c:499-760): data
 * scaling, x = argmin ||A x - y||^2 + lambda ||x||^2 by CG from zero
 * (conjgrad, src/iter/italgos.c:497-572). img is [X, Y, Z, 1]. */
int bnufft_pics_run(bnufft_pics_t pics, void* img, const void* ksp, void* stream);

/* Normal operator of the SENSE model, A^H A x (no lambda), img -> img. */
int bnufft_pics_normal(bnufft_pics_t pics, void* dst, const void* src, void* stream);

/* Statistics of the last run: iterations done, recursive relative residual
 * ||r||/||A^H y||, scaling used. Synchronises the stream. */
int bnufft_pics_stats(bnufft_pics_t pics, int* iters, double* rel_resid, float* scaling, void* stream);

/* Kernels the last run executed on the device: the ones launched from the
 * host plus those of the CG loop graph (its body once per iteration run).
 * Synchronises the stream. The CG loop runs as one CUDA graph with a while
 * node unless the environment sets BNUFFT_CG_GRAPH=0 (host loop, same
 * kernels and bit-identical results). */
int bnufft_pics_kernels(bnufft_pics_t pics, long* kernels, void* stream);

/* Releases the model without waiting for the device: its buffers are freed
 * in stream order after its last run, and its CG loop graph is kept for
 * the next model to reuse (or destroyed once that run has completed). */
void bnufft_pics_free(bnufft_pics_t pics);

/* Change the iteration limit and tolerance of later runs (the captured CG
 * graph reads them from the device, so it is kept). */
int bnufft_pics_set_iter(bnufft_pics_t pics, int maxiter, float tol);

/* Direct non-uniform DFT, replaces nudft_create / nudft_forward2 /
 * nudft_adjoint2 (src/noncart/nudft.c:69-348; `bart nufft -s`):
 * ksp[m, c] = s sum_n img[n, c] exp(-2 pi i k_m . (n - N/2) / N) and its
 * adjoint, s = 1 / sqrt(product of all image dims, coils included) as in the
 * reference. Same dims as bnufft_create2. No field map / time map. Exact
 * (float64-reduced phases), O(samples x pixels): for small sizes. */
typedef struct bnufft_nudft_s* bnufft_nudft_t;

int bnufft_nudft_create(bnufft_nudft_t* nudft, int N, const long ksp_dims[], const long cim_dims[],
		const long traj_dims[], const void* traj, void* stream);
int bnufft_nudft_apply_forward(bnufft_nudft_t nudft, void* ksp, const void* cim, void* stream);
int bnufft_nudft_apply_adjoint(bnufft_nudft_t nudft, void* cim, const void* ksp, void* stream);
void bnufft_nudft_free(bnufft_nudft_t nudft);

/* Batches (no counterpart in the reference, which runs one pics per problem,
 * src/pics.c, or loops with bart -p/-l, src/bart.c:202-217): n independent
 * models, each with its own size, trajectory, coil count and maps, and their
 * device k-space and image buffers, captured once into one CUDA graph in
 * which every problem's whole solve (scaling, CG with the model's fixed
 * maxiter, result) is an independent child graph; bnufft_batch_run launches
 * it, the problems run concurrently. Models and buffers must outlive the
 * batch; models need tol = 0. */
typedef struct bnufft_batch_s* bnufft_batch_t;

int bnufft_batch_create(bnufft_batch_t* batch, const bnufft_pics_t* models, int n, void* const* imgs,
		const void* const* ksps, void* stream);
int bnufft_batch_run(bnufft_batch_t batch, void* stream);
long bnufft_batch_kernels(bnufft_batch_t batch);	/* kernel nodes per launch */
void bnufft_batch_free(bnufft_batch_t batch);

/* b = A^H y / scale, the right-hand side the solve uses (scaling as in
 * bnufft_pics_run). img-sized output. */
int bnufft_pics_rhs(bnufft_pics_t pics, void* b, const void* ksp, void* stream);

/* z = M(r), the model's preconditioner (precond 1, 2 or 3) on one image. */
int bnufft_pics_precond(bnufft_pics_t pics, void* z, const void* r, void* stream);

/* Learned preconditioner (no counterpart in the reference; the reference's
 * plug-in point is the preconditioner operator of lsqr2_create,
 * src/iter/lsqr.c:126-143). A 6-layer 3x3 convolutional network,
 * 2 -> 32 -> 32 -> 32 -> 32 -> 32 -> 2 channels (complex image as 2
 * channels), ReLU after layers 1-5, bf16 weights and activations, float32
 * accumulation. Parameters: float32, per layer W[cout][3 ky + kx][cin] then
 * b[cout]; bnufft_precnet_nparams() values in all. Used by flexible CG as
 * z = M(r) + ||M(r)|| net(M(r) / ||M(r)||), M the padded-circulant
 * preconditioner. */
typedef struct bnufft_precnet_s* bnufft_precnet_t;

int bnufft_precnet_nparams(void);
int bnufft_precnet_create(bnufft_precnet_t* net, const float* params, void* stream);
int bnufft_precnet_set_params(bnufft_precnet_t net, const float* params, void* stream);
int bnufft_precnet_get_params(bnufft_precnet_t net, float* params, void* stream);

/* out = net(in) for nimg complex images [X, Y] (no scaling). */
int bnufft_precnet_forward(bnufft_precnet_t net, void* out, const void* in, long X, long Y, long nimg, void* stream);

/* One training step on a batch: loss = (1/nimg) sum |net(in) - target|^2,
 * its gradient (copied to grads if not null), then an Adam step with
 * learning rate lr (none if lr <= 0). loss (if not null) synchronises. */
int bnufft_precnet_train_step(bnufft_precnet_t net, const void* in, const void* target, long X, long Y, long nimg,
		float lr, double* loss, float* grads, void* stream);

/* The same step with the loss gradient d loss / d net(in) given by the
 * caller (gout, complex like in): for losses that need operators outside the
 * network. */
int bnufft_precnet_backward(bnufft_precnet_t net, const void* in, const void* gout, long X, long Y, long nimg,
		float lr, float* grads, void* stream);

/* The network's 32 -> 32 layers run on the tcgen05 tensor cores; their
 * waits for the tensor core are bounded. *status (synchronises): 0, or 1 if
 * a wait ran out since the network was created (the layer's output was then
 * not written). */
int bnufft_precnet_status(bnufft_precnet_t net, int* status, void* stream);

void bnufft_precnet_free(bnufft_precnet_t net);

/* Attach a network to a model created with precond 2 (not owned). */
int bnufft_pics_set_precnet(bnufft_pics_t pics, bnufft_precnet_t net, void* stream);

/* Host-only views of the library's interpolation tables (no device work,
 * usable without a GPU), built in float64 exactly as the plans build them:
 * bnufft_calc_beta replaces calc_beta (src/noncart/grid.c:516-519);
 * bnufft_kb_precompute replaces kb_precompute (src/noncart/grid.c:86-97,
 * table[i] = I0(beta sqrt(1 - (2x)^2)) / I0(beta), x = i / (n - 1) / 2, n + 1
 * floats; plans use n = 1000 and beta = float(calc_beta(os, width)), as
 * the reference's kb_init receives it from rolloff_correction);
 * bnufft_rolloff_axis gives the roll-off of one n-point image axis in
 * float64, rolloff(pos(n, i, os), beta, width) of src/noncart/grid.c:114-117,
 * 522-533. */
double bnufft_calc_beta(float os, float width);
int bnufft_kb_precompute(double beta, int n, float* table);
int bnufft_rolloff_axis(float os, float width, long n, double* roll);

/* CG on (A + lambda I) x = b for an operator A that the caller applies
 * between the calls, with the library's fused vector passes and its device
 * float64 scalars (the reference's conjgrad, src/iter/italgos.c:497-572;
 * f32_scalars: alpha, beta and the residual norms rounded to float as it
 * stores them). No counterpart in the reference: this is the solve of the
 * coil-sharded CG-SENSE, where A p is each GPU's coil share of the normal
 * operator summed by an all-reduce (its --md-split-mpi-dims with
 * mpi_reduce_zsum, src/num/mpi_ops.c:680-735). All vectors are device
 * arrays of n complex floats on the same stream.
 *   bnufft_cg_start: x = 0, r = b, p = z (z = M b for PCG, or NULL: b);
 *   per iteration, with q = A p (without lambda) from the caller:
 *   bnufft_cg_update: alpha = <r, z> / <p, q + lambda p>, x += alpha p,
 *     r -= alpha (q + lambda p);
 *   bnufft_cg_direction (z = M r for PCG, or NULL): stop when ||r|| <= tol
 *     ||b||, else p = z + beta p, beta = <r, z>_new / <r, z>_old.
 * Once stopped (or at p^H (A + lambda) p = 0) the calls leave x unchanged;
 * bnufft_cg_status reads (and synchronises on) the stop flag, the
 * iterations done and ||r||. */
typedef struct bnufft_cg_s* bnufft_cg_t;
int bnufft_cg_create(bnufft_cg_t* cg, long n, float lambda, float tol, int f32_scalars, void* stream);
int bnufft_cg_start(bnufft_cg_t cg, void* x, void* r, void* p, const void* b, const void* z, void* stream);
int bnufft_cg_update(bnufft_cg_t cg, void* x, void* r, const void* p, const void* q, void* stream);
int bnufft_cg_direction(bnufft_cg_t cg, void* p, const void* r, const void* z, void* stream);
int bnufft_cg_status(bnufft_cg_t cg, int* done, int* iters, float* rnorm, void* stream);
void bnufft_cg_free(bnufft_cg_t cg);

/* Message of the last failure on this thread ("" if none). */
const char* bnufft_last_error(void);

/* Number of kernel launches issued by this library since load. */
long bnufft_launch_count(void);

/* Instrumentation (no counterpart in the reference): time every launch of
 * one kernel class ("rows_fwd", "cols_fwd", "cols_inv", "cols_toeplitz",
 * "rows_inv", "degrid", "grid"; the passes of the circulant preconditioner
 * as "precond_rows_fwd", "precond_cols_toeplitz", "precond_rows_inv") with
 * CUDA events on its stream until
 * bnufft_prof_stop(), which returns the summed device time and launch count. */
int bnufft_prof_start(const char* kind);
int bnufft_prof_stop(double* total_ms, long* launches);

#ifdef __cplusplus
}
#endif
#endif
