// Vector kernels of the CG-SENSE solve, fused into single passes.
//
// The reference runs CG (src/iter/italgos.c:497-572) with one kernel per
// vector op and a device->host copy for every dot product
// (src/num/gpuops.c:633-665). Here the scalars stay on the device in float64:
// each pass writes per-block float64 partial sums, and the next pass reduces
// them in a fixed order (every block redundantly), so the iteration needs no
// host synchronisation and the sums are bit-reproducible run to run.
#pragma once

#include <cuda_runtime.h>

#include "fft_core.cuh"
#include "nufft_kernels.cuh"

namespace bn {

// sum of the coil-group partials part[i + n g], g = 0..groups-1, in order;
// the loads of eight groups at a time are issued together
__device__ __forceinline__ float2 group_sum(const float2* __restrict__ part, long i, long n, int groups)
{
	float2 v = part[i];

	for (int g0 = 1; g0 < groups; g0 += 8) {

		float2 t[8];
#pragma unroll
		for (int k = 0; k < 8; k++)
			t[k] = (g0 + k < groups) ? part[i + n * (g0 + k)] : make_float2(0.f, 0.f);
#pragma unroll
		for (int k = 0; k < 8; k++)
			if (g0 + k < groups)
				v = cadd(v, t[k]);
	}

	return v;
}

enum { RED_THREADS = 256 };

template <typename T>
__device__ __forceinline__ T block_sum(T v, T* sh)
{
	for (int o = 16; o > 0; o >>= 1)
		v += __shfl_down_sync(0xffffffffu, v, o);

	int w = threadIdx.x / 32;
	int l = threadIdx.x % 32;

	if (0 == l)
		sh[w] = v;

	__syncthreads();

	T r = 0;

	if (threadIdx.x < 32) {

		r = (threadIdx.x < blockDim.x / 32) ? sh[threadIdx.x] : (T)0;

		for (int o = 16; o > 0; o >>= 1)
			r += __shfl_down_sync(0xffffffffu, r, o);
	}

	return r;	// valid in thread 0
}

__device__ __forceinline__ double sum_partials(const double* part, int n, double* sh)
{
	return sum_partials_d(part, n, sh);
}

// dst[i] = sum_g part[i + n*g] (+ lam * x[i]); optional per-block partial of
// Re<x, dst> into dot_part. n complex elements.
__global__ void k_combine(float2* __restrict__ dst, const float2* __restrict__ part, int groups, long n,
		const float2* __restrict__ x, float lam, double* __restrict__ dot_part, const int* done)
{
	__shared__ double sh[32];

	if (done && *done)
		return;

	double acc = 0.;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		float2 v = group_sum(part, i, n, groups);

		if (x) {

			float2 xv = x[i];
			v.x = fmaf(lam, xv.x, v.x);
			v.y = fmaf(lam, xv.y, v.y);
			acc += (double)xv.x * (double)v.x + (double)xv.y * (double)v.y;
		}

		dst[i] = v;
	}

	if (dot_part) {

		double r = block_sum(acc, sh);

		if (0 == threadIdx.x)
			dot_part[blockIdx.x] = r;
	}
}

// CG start from x = 0: x = 0, r = p = b; partial ||b||^2.
__global__ void k_cg_init(float2* __restrict__ x, float2* __restrict__ r, float2* __restrict__ p,
		const float2* __restrict__ b, long n, double* __restrict__ part)
{
	__shared__ double sh[32];
	double acc = 0.;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		float2 v = b[i];
		x[i] = make_float2(0.f, 0.f);
		r[i] = v;
		p[i] = v;
		acc += (double)v.x * (double)v.x + (double)v.y * (double)v.y;
	}

	double s = block_sum(acc, sh);

	if (0 == threadIdx.x)
		part[blockIdx.x] = s;
}

// rs[0] = ||b||^2 = b2, eps2 = (tol*||b||)^2, iters = 0, done = (b2 == 0).
// f32: the plain CG's scalars in float32 as the reference keeps them:
// eps = float(||b||) * tol and eps2 = float(eps^2) (iter2_conjgrad,
// src/iter/iter2.c:249-254; conjgrad, src/iter/italgos.c:518-523).
__global__ void k_cg_start(CgScalars* st, const double* part, int nparts, float tol, int maxiter, int f32,
		int net_iters = 0)
{
	__shared__ double sh[32];
	double b2 = sum_partials(part, nparts, sh);

	if (0 == threadIdx.x) {

		st->f32 = f32;
		st->b2 = b2;
		st->rs[0] = cg_keep(st, b2);

		if (f32) {

			float eps = __fmul_rn((float)sqrt(b2), tol);
			st->eps2 = (double)(float)((double)eps * (double)eps);

		} else {

			double eps = (double)tol * sqrt(b2);
			st->eps2 = eps * eps;
		}

		st->iters = 0;
		st->it = 0;
		st->maxiter = maxiter;
		st->done = (0. == b2);
		st->best_rs = b2;
		st->best_hist[0] = b2;
		st->best_it = 0;
		st->net_off = 0;
		st->net_iters = net_iters;
		st->restart_it = 0;
		st->rnorm = (float)sqrt(b2);
		st->rinv = (b2 > 0.) ? (float)(1. / sqrt(b2)) : 0.f;
	}
}

// Second step of a CG iteration: p^H (A^H A + lambda) p from the partials of
// the last row pass and of ||p||^2; alpha = rs / p^H A p (float64); then per
// element Ap = sum_g part_g + lambda p, x += alpha p, r -= alpha Ap, and
// partial ||r||^2 for the next iteration's direction update. p is also
// copied to p_keep (the next iteration's previous direction) when given.
__global__ void k_cg_step(float2* __restrict__ x, float2* __restrict__ r, const float2* __restrict__ p,
		const float2* __restrict__ part, int groups, long n, float lam, CgScalars* st, int it,
		const double* __restrict__ pap_part, int npap, const double* __restrict__ pp_part, int npp,
		double* __restrict__ rs_part, float2* __restrict__ p_keep)
{
	__shared__ double sh[96];

	if (st->done)
		return;

	it = cg_iter(it, st);
	const double3 sums = sum_partials3_d(pap_part, npap, pp_part, npp, nullptr, 0, sh);
	double pAp = cg_keep(st, sums.x + (double)lam * sums.y);

	if (0. == pAp) {

		if ((0 == blockIdx.x) && (0 == threadIdx.x)) {

			st->done = 1;
			st->iters = it;
		}

		return;
	}

	float a = cg_ratio(st, st->rs[it & 1], pAp);
	double acc = 0.;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		float2 pv = p[i];
		float2 av = group_sum(part, i, n, groups);

		if (p_keep)
			p_keep[i] = pv;

		av.x = fmaf(lam, pv.x, av.x);
		av.y = fmaf(lam, pv.y, av.y);

		float2 xv = x[i];
		float2 rv = r[i];
		xv.x = fmaf(a, pv.x, xv.x);
		xv.y = fmaf(a, pv.y, xv.y);
		rv.x = fmaf(-a, av.x, rv.x);
		rv.y = fmaf(-a, av.y, rv.y);
		x[i] = xv;
		r[i] = rv;
		acc += (double)rv.x * (double)rv.x + (double)rv.y * (double)rv.y;
	}

	double s = block_sum(acc, sh);

	if (0 == threadIdx.x)
		rs_part[blockIdx.x] = s;
}

// Direction update of the plain CG (conjgrad, src/iter/italgos.c:558-566):
// rs_new = ||r||^2 from the step's partials; stop if rs_new <= eps2, else
// p = r + (rs_new / rs_old) p. rs of iteration it+1 goes to rs[(it+1) & 1].
__global__ void k_cg_dir(float2* __restrict__ p, const float2* __restrict__ r, long n, CgScalars* st, int it,
		const double* __restrict__ rs_part, int nrs)
{
	__shared__ double sh[32];

	if (st->done)
		return;

	double rs_new = cg_keep(st, sum_partials(rs_part, nrs, sh));
	double rs_old = st->rs[it & 1];
	bool stop = (rs_new <= st->eps2);

	if (!stop) {

		float beta = cg_ratio(st, rs_new, rs_old);

		for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

			float2 pv = p[i];
			float2 rv = r[i];
			pv.x = fmaf(beta, pv.x, rv.x);
			pv.y = fmaf(beta, pv.y, rv.y);
			p[i] = pv;
		}
	}

	if ((0 == blockIdx.x) && (0 == threadIdx.x)) {

		st->rs[(it + 1) & 1] = rs_new;
		st->iters = it + 1;

		if (stop)
			st->done = 1;
	}
}

// The padded-circulant preconditioner (no counterpart in the reference):
// the Toeplitz normal operator is T = crop F^-1 P F pad on its power-of-two
// grid, and M^-1 = crop F^-1 (|P| + mu)^-1 F pad inverts that circulant
// on the padded image instead of the reference's N-point (Strang)
// circulant. mu = max(mu_lam, 1e-3 |P_0|) (P_0 the spectrum's DC value,
// index 0 in DFT order): mu_lam = 2.5 lambda 4^d / (grid cells) was the
// best multiple of lambda on FP64 oracle solves of 2D radial problems
// (35-45 % fewer iterations to 1e-4 than the Strang preconditioner).
__global__ void k_precond_pad_spectrum(float2* __restrict__ pinv, const float2* __restrict__ psf, long n, float mu_lam)
{
	const float2 p0 = psf[0];
	const float mu = fmaxf(mu_lam, 1e-3f * hypotf(p0.x, p0.y));

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		float2 v = psf[i];
		pinv[i] = make_float2(1.f / (hypotf(v.x, v.y) + mu), 0.f);
	}
}

// 1 / (|F| / sqrt(npix) + 1e-3) as a complex multiplier: the reference's
// circulant preconditioner (compute_precond, src/noncart/precond.c:56-60)
// from the N-point spectrum F of its kernel
__global__ void k_precond_from_spectrum(float2* __restrict__ pinv, const float2* __restrict__ F, long n, float inv_sqrt_npix)
{
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		float2 v = F[i];
		float pre = hypotf(v.x, v.y) * inv_sqrt_npix + 1e-3f;
		pinv[i] = make_float2(1.f / pre, 0.f);
	}
}

// Flexible CG (Notay, SIAM J. Sci. Comput. 22(4), 2000) with truncation m:
// the preconditioner z = M(r) may be nonlinear (the learned one), so each new
// direction is made A-orthogonal to the last m directions,
//   p_k = z_k - sum_{j = k-m}^{k-1} (<z_k, A p_j> / <p_j, A p_j>) p_j,
//   alpha = <p_k, r_k> / <p_k, A p_k>,  x += alpha p_k,  r -= alpha A p_k.
// The last FCG_RING directions and their A p live in ring buffers
// [FCG_RING][n], slot j % FCG_RING, indexed from the device iteration counter.

// partials of <z, A p_j> for the window j = it - w .. it - 1,
// w = min(it - restart, m) (the history restarts when the preconditioner changes):
// part[q * gridDim.x + block], q = j - (it - w)
__global__ void k_fcgm_dots(const float2* __restrict__ z, const float2* __restrict__ ap_ring, long n,
		const CgScalars* st, int it, int m, int ring, double* __restrict__ part)
{
	__shared__ double sh[32];

	if (st->done)
		return;

	it = cg_iter(it, st);
	const int w = min(it - st->restart_it, m);
	double acc[FCG_MAX_M];
#pragma unroll
	for (int q = 0; q < FCG_MAX_M; q++)
		acc[q] = 0.;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		float2 zv = z[i];
#pragma unroll
		for (int q = 0; q < FCG_MAX_M; q++) {

			if (q < w) {

				float2 a = ap_ring[(long)((it - w + q) % ring) * n + i];
				acc[q] += (double)zv.x * (double)a.x + (double)zv.y * (double)a.y;
			}
		}
	}

#pragma unroll
	for (int q = 0; q < FCG_MAX_M; q++) {

		if (q < w) {

			double t = block_sum(acc[q], sh);

			if (0 == threadIdx.x)
				part[q * gridDim.x + blockIdx.x] = t;

			__syncthreads();
		}
	}
}

// direction: p = z - sum_q beta_q p_{it-w+q}; p into p_cur and ring slot
// it % FCG_RING; partials <p, r> and ||p||^2 (lambda ||p||^2 in <p, A p>)
__global__ void k_fcgm_dir(float2* __restrict__ p_cur, float2* __restrict__ p_ring, const float2* __restrict__ z,
		const float2* __restrict__ r, long n, CgScalars* st, int it, int m, int ring, const double* __restrict__ dots,
		int ndots, double* __restrict__ pr_part, double* __restrict__ pp_part, const double* __restrict__ rs_part, int nrs)
{
	__shared__ double sh[96];
	__shared__ float beta[FCG_MAX_M];

	if (st->done)
		return;

	it = cg_iter(it, st);
	// the learned term's iteration budget: z of iterations < net_iters
	// carries it, and the first direction after it restarts (p = z, PCG
	// from there on; a short recurrence across the switch converges slower).
	// Every block derives the restart from it alone; net_off is only read
	// by the preconditioner pass at the end of this iteration (z for
	// iteration it + 1).
	const bool restart = (st->net_iters > 0) && (it == st->net_iters);
	const int w = restart ? 0 : min(it - st->restart_it, m);
	const bool check = rs_part && (it > 0);

	if ((0 == blockIdx.x) && (0 == threadIdx.x) && (st->net_iters > 0) && (it + 1 >= st->net_iters))
		st->net_off = 1;
	// ||r||^2 and the first <z, A p_j> in one reduction
	const double3 s3 = sum_partials3_d(rs_part, check ? nrs : 0, dots, (w > 0) ? ndots : 0, nullptr, 0, sh);

	// with rs_part: the convergence test of the previous step is done here
	// (every block reaches the same decision from the same partial sums)
	if (check) {

		double rs = s3.x;

		if ((0 == blockIdx.x) && (0 == threadIdx.x)) {

			st->rs[it & 1] = rs;

			if (rs <= st->eps2) {

				st->done = 1;
				st->iters = it;
			}
		}

		if (rs <= st->eps2)
			return;
	}

	for (int q = 0; q < w; q++) {

		double d = (0 == q) ? s3.y : sum_partials(dots + q * ndots, ndots, sh);

		if (0 == threadIdx.x)
			beta[q] = (float)(d / st->pap_hist[(it - w + q) % ring]);
	}

	__syncthreads();

	float2* p_slot = p_ring + (long)(it % ring) * n;
	double pr = 0., pp = 0.;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		float2 pv = z[i];

		for (int q = 0; q < w; q++) {

			float2 o = p_ring[(long)((it - w + q) % ring) * n + i];
			pv.x = fmaf(-beta[q], o.x, pv.x);
			pv.y = fmaf(-beta[q], o.y, pv.y);
		}

		p_cur[i] = pv;
		p_slot[i] = pv;
		float2 rv = r[i];
		pr += (double)pv.x * (double)rv.x + (double)pv.y * (double)rv.y;
		pp += (double)pv.x * (double)pv.x + (double)pv.y * (double)pv.y;
	}

	double t = block_sum(pr, sh);
	__syncthreads();
	double u = block_sum(pp, sh);

	if (0 == threadIdx.x) {

		pr_part[blockIdx.x] = t;
		pp_part[blockIdx.x] = u;
	}
}

// FCG step: <p, A p> (coil-sum row-pass partials + lambda ||p||^2), alpha =
// <p, r> / <p, A p>; per element A p = sum_g part_g + lambda p (into ring
// slot it % FCG_RING), x += alpha p, r -= alpha A p, partial ||r||^2.
__global__ void k_fcg_step(float2* __restrict__ x, float2* __restrict__ r, const float2* __restrict__ p,
		float2* __restrict__ ap_ring, int ring, const float2* __restrict__ part, int groups, long n, float lam, CgScalars* st, int it,
		const double* __restrict__ pap_part, int npap, const double* __restrict__ pp_part, int npp,
		const double* __restrict__ pr_part, int npr, double* __restrict__ rs_part)
{
	__shared__ double sh[96];

	if (st->done)
		return;

	it = cg_iter(it, st);
	const double3 sums = sum_partials3_d(pap_part, npap, pp_part, npp, pr_part, npr, sh);
	double pAp = sums.x + (double)lam * sums.y;

	if (!(pAp > 0.)) {	// zero or not positive: breakdown

		if ((0 == blockIdx.x) && (0 == threadIdx.x)) {

			st->done = 1;
			st->iters = it;
		}

		return;
	}

	float a = (float)(sums.z / pAp);
	float2* Ap = ap_ring + (long)(it % ring) * n;
	double acc = 0.;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		float2 pv = p[i];
		float2 av = group_sum(part, i, n, groups);

		av.x = fmaf(lam, pv.x, av.x);
		av.y = fmaf(lam, pv.y, av.y);
		Ap[i] = av;

		float2 xv = x[i];
		float2 rv = r[i];
		xv.x = fmaf(a, pv.x, xv.x);
		xv.y = fmaf(a, pv.y, xv.y);
		rv.x = fmaf(-a, av.x, rv.x);
		rv.y = fmaf(-a, av.y, rv.y);
		x[i] = xv;
		r[i] = rv;
		acc += (double)rv.x * (double)rv.x + (double)rv.y * (double)rv.y;
	}

	double s = block_sum(acc, sh);

	if (0 == threadIdx.x)
		rs_part[blockIdx.x] = s;

	if ((0 == blockIdx.x) && (0 == threadIdx.x))
		st->pap_hist[it % ring] = pAp;
}

// FCG convergence test after step it: ||r||^2 <= eps2 stops with it + 1
// iterations done
__global__ void k_fcg_check(CgScalars* st, int it, const double* __restrict__ rs_part, int nrs)
{
	__shared__ double sh[32];

	if (st->done)
		return;

	it = cg_iter(it, st);
	double rs = sum_partials(rs_part, nrs, sh);

	if (0 == threadIdx.x) {

		st->rs[(it + 1) & 1] = rs;
		st->rnorm = (float)sqrt(rs);
		st->rinv = (rs > 0.) ? (float)(1. / sqrt(rs)) : 0.f;

		if (rs <= st->eps2) {

			st->done = 1;
			st->iters = it + 1;
		}

		// stall: no new smallest residual for 3 iterations, or less than a 4x
		// reduction of the smallest ||r||^2 over the last 4 iterations,
		// switches the learned part of the preconditioner off for the rest
		// of the solve (the method falls back to its linear preconditioner)
		const int j = it + 1;

		if (rs < st->best_rs) {

			st->best_rs = rs;
			st->best_it = j;

		}

		bool stall = (j - st->best_it >= 3) || ((j >= 4) && (st->best_rs > 0.25 * st->best_hist[j % 4]));

		// the learned part's iteration budget: once it is spent the
		// preconditioner is the linear one, and the direction history
		// restarts (one kept direction from here on, as PCG)
		if ((st->net_iters > 0) && (j >= st->net_iters) && !st->net_off) {

			st->net_off = 1;
			st->restart_it = j;
		}

		if (stall && !st->net_off) {

			// the preconditioner changes: restart the direction history
			st->net_off = 1;
			st->restart_it = j;
		}

		st->best_hist[j % 4] = st->best_rs;
	}
}

// ||v|| into the scalars (rnorm, rinv) for a preconditioner applied outside
// a solve; clears done and the stall flag
__global__ void k_norm_scalars(const float2* __restrict__ v, long n, CgScalars* st)
{
	__shared__ double sh[32];
	double acc = 0.;

	for (long i = threadIdx.x; i < n; i += blockDim.x)
		acc += (double)v[i].x * v[i].x + (double)v[i].y * v[i].y;

	double s = block_sum(acc, sh);

	if (0 == threadIdx.x) {

		st->rnorm = (float)sqrt(s);
		st->rinv = (s > 0.) ? (float)(1. / sqrt(s)) : 0.f;
		st->done = 0;
		st->net_off = 0;
		st->restart_it = 0;
	}
}

// End of one CG iteration inside a graph: advance the device iteration
// counter and continue the enclosing while node unless converged or at maxiter.
__global__ void k_cg_advance(CgScalars* st, cudaGraphConditionalHandle loop)
{
	int it = st->it + 1;
	st->it = it;
	cudaGraphSetConditional(loop, (!st->done && (it < st->maxiter)) ? 1u : 0u);
}

// after the last iteration: ||r||^2 and the iteration count
__global__ void k_cg_finish(CgScalars* st, int maxiter, const double* rs_part, int nrs)
{
	__shared__ double sh[32];

	if (st->done)
		return;

	double rs = sum_partials(rs_part, nrs, sh);

	if (0 == threadIdx.x) {

		st->rs[maxiter & 1] = rs;
		st->iters = maxiter;
	}
}

// dst = src * scalar (scalar read from device memory, float)
__global__ void k_scale_dev(float2* __restrict__ dst, const float2* __restrict__ src, long n, const float* s)
{
	float f = *s;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
		dst[i] = cscale(src[i], f);
}

__global__ void k_scale(float2* __restrict__ dst, const float2* __restrict__ src, long n, float f)
{
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
		dst[i] = cscale(src[i], f);
}

// estimate_scaling_norm (src/sense/optcom.c:74-109): of the magnitudes |b|
// sorted ascending, p90 unless (max - p90) >= 2 (p90 - median), then max;
// 0 -> 1. The three order statistics (ranks n/2, trunc(0.9 n), n - 1) come
// without sorting from a radix select over the magnitudes' bit
// patterns (non-negative floats order like their unsigned bits) in three
// passes of 11, 11 and 10 bits. Each pass histograms the digit of the
// elements whose higher bits match a rank's prefix so far (one shared
// histogram in the first pass), the counts are added into the state with
// integer atomics (exact, order-free), and the last block to finish picks
// each rank's digit and resets the histograms. The third pass ends with the
// three values, exactly the sorted array's entries.
enum { SEL_BINS = 2048, SEL_THREADS = 256 };

struct SelectState {

	alignas(16) unsigned hist[3][SEL_BINS];	// first: 16-byte vector access
	unsigned prefix[3];	// key bits chosen so far per rank
	long long rank[3];	// rank left within the chosen prefix
	unsigned blocks_done;
};

template <int P>
struct SelDigit {

	static constexpr int SHIFT = (0 == P) ? 21 : ((1 == P) ? 10 : 0);
	static constexpr int W = (2 == P) ? 10 : 11;
};

template <int P>
__global__ void __launch_bounds__(SEL_THREADS) k_select_pass(const float2* __restrict__ b, float* __restrict__ mag,
		long n, SelectState* ss, CgScalars* st)
{
	constexpr int SHIFT = SelDigit<P>::SHIFT;
	constexpr int W = SelDigit<P>::W;
	constexpr int NB = 1 << W;
	constexpr int NH = (0 == P) ? 1 : 3;
	__shared__ __align__(16) unsigned h[NH * NB];
	__shared__ unsigned pre[3];
	__shared__ int last;

	for (int i = threadIdx.x; i < NH * NB; i += blockDim.x)
		h[i] = 0u;

	if (threadIdx.x < 3)
		pre[threadIdx.x] = ss->prefix[threadIdx.x];

	__syncthreads();

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		float m;

		if (0 == P) {

			float2 v = b[i];
			m = hypotf(v.x, v.y);	// cabsf
			mag[i] = m;

		} else {

			m = mag[i];
		}

		const unsigned key = __float_as_uint(m);
		const unsigned d = (key >> SHIFT) & (NB - 1);

		if (0 == P) {

			atomicAdd(&h[d], 1u);

		} else {
#pragma unroll
			for (int j = 0; j < 3; j++)
				if ((key >> (SHIFT + W)) == (pre[j] >> (SHIFT + W)))
					atomicAdd(&h[j * NB + d], 1u);
		}
	}

	__syncthreads();

	for (int i = threadIdx.x; i < NH * NB; i += blockDim.x)
		if (h[i])
			atomicAdd(&ss->hist[0][0] + i, h[i]);

	__threadfence();
	__syncthreads();

	if (0 == threadIdx.x)
		last = (atomicAdd(&ss->blocks_done, 1u) == gridDim.x - 1);

	__syncthreads();

	if (!last)
		return;

	__threadfence();

	// the global histograms into shared memory (16-byte loads from L2)
	for (int i = threadIdx.x; i < NH * NB / 4; i += blockDim.x)
		reinterpret_cast<uint4*>(h)[i] = __ldcg(reinterpret_cast<const uint4*>(&ss->hist[0][0]) + i);

	__syncthreads();
	const int warp = threadIdx.x / 32;
	const int lane = threadIdx.x % 32;

	if (warp < 3) {	// one warp per rank: the digit holding it

		const unsigned* hg = h + ((0 == P) ? 0 : warp * NB);
		long long rank = (0 == P) ? ((0 == warp) ? n / 2 : ((1 == warp) ? (long long)trunc(n * 0.9) : n - 1))
					  : ss->rank[warp];
		constexpr int PER = NB / 32;
		unsigned tot = 0u;

		for (int k = 0; k < PER; k++)
			tot += hg[lane * PER + k];

		unsigned incl = tot;

		for (int o = 1; o < 32; o <<= 1) {

			unsigned t = __shfl_up_sync(0xffffffffu, incl, o);

			if (lane >= o)
				incl += t;
		}

		const long long excl = (long long)incl - tot;
		const bool mine = (excl <= rank) && (rank < (long long)incl);

		if (mine) {

			long long before = excl;
			int dsel = lane * PER;

			for (int k = 0; k < PER; k++) {

				unsigned c = hg[lane * PER + k];

				if (rank < before + (long long)c) {

					dsel = lane * PER + k;
					break;
				}

				before += c;
			}

			const unsigned base = (0 == P) ? 0u : pre[warp];
			ss->prefix[warp] = base | ((unsigned)dsel << SHIFT);
			ss->rank[warp] = rank - before;
		}
	}

	__syncthreads();

	for (int i = threadIdx.x; i < NH * NB / 4; i += blockDim.x)
		reinterpret_cast<uint4*>(&ss->hist[0][0])[i] = make_uint4(0u, 0u, 0u, 0u);

	if (0 == threadIdx.x) {

		ss->blocks_done = 0u;

		if (2 == P) {	// estimate_scaling_norm

			float median = __uint_as_float(ss->prefix[0]);
			float p90 = __uint_as_float(ss->prefix[1]);
			float mx = __uint_as_float(ss->prefix[2]);
			float scale = ((mx - p90) < 2 * (p90 - median)) ? p90 : mx;

			if (0.f == scale)
				scale = 1.f;

			st->scale = scale;
			st->inv_scale = (float)(1. / scale);
		}
	}
}

__global__ void k_set_scaling(CgScalars* st, float scale)
{
	st->scale = scale;
	st->inv_scale = (float)(1. / scale);
}

__global__ void k_fill(float2* dst, long n, float2 v)
{
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
		dst[i] = v;
}

// y[m + M*c] = x[m + M*c] * w[m + M*(c % cw)] (conj(w) when conj): density
// weights / sampling pattern of the NUFFT (src/noncart/nufft.c:1456, 1474)
__global__ void k_weight(float2* __restrict__ y, const float2* __restrict__ x, const float2* __restrict__ w,
		long M, long C, long cw, int conj)
{
	long n = M * C;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		long m = i % M;
		long c = i / M;
		float2 wv = w[m + M * (c % cw)];
		y[i] = conj ? cmulc(x[i], wv) : cmul(x[i], wv);
	}
}

// |w|^2 (real) into a complex buffer: the PSF's "ones" with weights
__global__ void k_weight_sq(float2* __restrict__ y, const float2* __restrict__ w, long M)
{
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (long)gridDim.x * blockDim.x) {

		float2 v = w[i];
		y[i] = cmulc(v, v);
	}
}

// trajectory [3, M] complex float -> float4 (kx, ky, kz, 0) * factor
__global__ void k_traj_convert(float4* __restrict__ dst, const float2* __restrict__ src, long M, float factor)
{
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (long)gridDim.x * blockDim.x)
		dst[i] = make_float4(src[3 * i + 0].x * factor, src[3 * i + 1].x * factor, src[3 * i + 2].x * factor, 0.f);
}

// Subspace basis (nufft_create2 with a basis, src/noncart/nufft.c:1427-1491,
// 1546-1625). Samples of all T frames form one list of Mt = MrMs * T samples
// (frame t at [t MrMs, (t + 1) MrMs)); the NUFFT's channels are (c, k), c <
// Cc coils, k < K coefficients, channel c + Cc k; k-space is the
// reference's [1, Mr, Ms, Cc, 1, T] array, element m + MrMs (c + Cc t); the
// basis [1, 1, 1, 1, 1, T, K], element t + T k.

// forward: ksp[m, c, t] = sum_k B[t, k] tmp[t MrMs + m, c + Cc k]
// (md_ztenmul over COEFF, :1450-1453)
__global__ void k_basis_contract(float2* __restrict__ ksp, const float2* __restrict__ tmp, const float2* __restrict__ B,
		long MrMs, int T, long Cc, int K)
{
	const long Mt = MrMs * T;
	const long n = Mt * Cc;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		const long m = i % MrMs;
		const long c = (i / MrMs) % Cc;
		const int t = (int)(i / (MrMs * Cc));
		float2 acc = make_float2(0.f, 0.f);

		for (int k = 0; k < K; k++) {

			const float2 v = tmp[t * MrMs + m + Mt * (c + Cc * k)];
			const float2 b = B[t + (long)T * k];
			acc.x = fmaf(b.x, v.x, fmaf(-b.y, v.y, acc.x));
			acc.y = fmaf(b.x, v.y, fmaf(b.y, v.x, acc.y));
		}

		ksp[i] = acc;
	}
}

// adjoint: tmp[t MrMs + m, c + Cc k] = conj(B[t, k]) ksp[m, c, t]
// (md_ztenmulc, :1483-1487)
__global__ void k_basis_expand(float2* __restrict__ tmp, const float2* __restrict__ ksp, const float2* __restrict__ B,
		long MrMs, int T, long Cc, int K)
{
	const long Mt = MrMs * T;
	const long n = Mt * Cc * K;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		const long mt = i % Mt;			// t MrMs + m
		const long ch = i / Mt;			// c + Cc k
		const long c = ch % Cc;
		const int k = (int)(ch / Cc);
		const int t = (int)(mt / MrMs);
		const long m = mt % MrMs;
		tmp[i] = cmulc(ksp[m + MrMs * (c + Cc * t)], B[t + (long)T * k]);
	}
}

// the PSF's k-space for coefficient pair j = k + K k' (compute_square_basis
// and the adjoint's conjugate, :470-505, 535-586):
// w[s, j] = conj(B[t(s), k]) B[t(s), k'] |wgt[s]|^2 (wgt: Mt sample weights or null)
__global__ void k_basis_psf_weights(float2* __restrict__ w, const float2* __restrict__ B,
		const float2* __restrict__ wgt, long MrMs, int T, int K)
{
	const long Mt = MrMs * T;
	const long n = Mt * K * K;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		const long s = i % Mt;
		const int j = (int)(i / Mt);
		const int k = j % K, kp = j / K;
		const int t = (int)(s / MrMs);
		float2 v = cmulc(B[t + (long)T * kp], B[t + (long)T * k]);

		if (wgt) {

			const float2 u = wgt[s];
			const float a = u.x * u.x + u.y * u.y;
			v = make_float2(v.x * a, v.y * a);
		}

		w[i] = v;
	}
}

enum { BASIS_MAX_K = 32 };

// the block-Toeplitz product on the spectrum (md_ztenmul with the psf
// [K (out)][K (in)], :1586-1592): spec[g, c + Cc k] <- sum_k'
// P[g, k + K k'] spec[g, c + Cc k'], for every cell g < gsz and coil c
__global__ void k_basis_mix(float2* __restrict__ spec, const float2* __restrict__ P, long gsz, long Cc, int K)
{
	const long n = gsz * Cc;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		const long g = i % gsz;
		const long c = i / gsz;
		float2 x[BASIS_MAX_K];

		for (int k = 0; k < K; k++)
			x[k] = spec[g + gsz * (c + Cc * k)];

		for (int k = 0; k < K; k++) {

			float2 acc = make_float2(0.f, 0.f);

			for (int kp = 0; kp < K; kp++) {

				const float2 pv = P[g + gsz * (k + (long)K * kp)];
				acc.x = fmaf(pv.x, x[kp].x, fmaf(-pv.y, x[kp].y, acc.x));
				acc.y = fmaf(pv.x, x[kp].y, fmaf(pv.y, x[kp].x, acc.y));
			}

			spec[g + gsz * (c + Cc * k)] = acc;
		}
	}
}

} // namespace bn
