// The circulant preconditioner of a 2D image in one launch on one thread-block
// cluster (nufft_precond_create / its apply, src/noncart/precond.c:36-64,
// 95-130; the spectrum pinv as built by build_precond):
//   z = IFFT_cols(pinv . FFT_cols(FFT_rows(r))) followed by IFFT_rows,
// N-point transforms with the centred placement (pixel x at position
// (x - N/2) mod N on both axes), exactly the arithmetic of the three-pass
// form (k_rows_fwd, k_cols mode 2, k_rows_inv) with the same FFT core and
// twiddles, so z is bit-identical to it.
//
// Cluster of CL CTAs (16 where the device allows that non-portable size,
// else 8); CTA c owns image rows [c R, (c + 1) R), R = N / CL, in shared
// memory (rowbuf). N / 8 threads serve one sequence, so a CTA has R * N / 8
// threads and R sequences in each phase:
//   1. forward FFT of its R rows into its rowbuf; cluster barrier
//   2. columns [c R, (c + 1) R): each thread loads its eight column elements
//      from the owners' rowbufs (distributed shared memory; a warp reads
//      consecutive columns of a row), forward FFT, * pinv (loaded before the
//      transform), inverse FFT, stores them back where it read them (no other
//      CTA touches these columns); cluster barrier
//   3. inverse FFT of its own rows from its rowbuf, uncentred output z and
//      the partial <pdot, z> of the CTA (flexible CG's next beta).
// After the second barrier no CTA touches another's shared memory, so CTAs
// may exit independently.
//
// With PcDir (flexible CG with one kept direction) the kernel also ends the
// CG iteration: before the transforms, the convergence test of the step
// just taken (||r||^2 partials; every CTA reaches the same decision, so all
// return together); after them, <A p, z> is summed over the CTAs through
// distributed shared memory in a fixed order, beta = <A p, z> / <p, A p>,
// p = z - beta p in place (p = z for the first direction), and per CTA the
// partials <p, r> and ||p||^2 of the next step. z itself is not stored.
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "fft_core.cuh"
#include "nufft_kernels.cuh"

namespace bn {

struct PcDir {

	CgScalars* st;		// nullptr: plain application
	int it;			// the step just taken (< 0: the device counter)
	int start;		// first direction: p = z, no test
	const double* rs_part;	// ||r||^2 partials of the step
	int nrs;
	float2* p;		// the direction, updated in place
	const float2* r;	// the residual
	double* pr_part;	// [CL] partials <p, r>
	double* pp_part;	// [CL] partials ||p||^2
};

template <int N, int CL>
struct PrecondClusterShape {

	static constexpr int R = N / CL;	// rows (and columns) per CTA
	static constexpr int T = N / 8;		// threads per sequence
	static constexpr int NT = R * T;	// threads per CTA
	using RL = RowLayout<N, R>;
	using CLY = ColLayout<N, R>;
	static constexpr int SCR = (RL::SMEM > CLY::SMEM) ? RL::SMEM : CLY::SMEM;
	static constexpr size_t SMEM = sizeof(float2) * ((size_t)R * N + SCR + N);
	static_assert((NT % 32 == 0) && (NT <= 1024), "whole warps, one CTA per SM");
};

// launched as one cluster of CL CTAs (cluster dimension given at launch)
template <int N, int CL>
__global__ void __launch_bounds__(PrecondClusterShape<N, CL>::NT, 1)
k_precond_cluster(const float2* __restrict__ r, const float2* __restrict__ pinv, float2* z,
		const float2* __restrict__ twg, const float2* pdot, double* __restrict__ dot_part, const int* done,
		PcDir dir)
{
	using S = PrecondClusterShape<N, CL>;
	constexpr int R = S::R;
	constexpr int T = S::T;
	using RL = typename S::RL;
	using CLY = typename S::CLY;
	extern __shared__ float2 smem[];
	__shared__ double red[32];
	__shared__ double cdot;
	float2* rowbuf = smem;			// [R][N] this CTA's rows
	float2* s = smem + R * N;		// FFT scratch
	float2* tw = s + S::SCR;

	// done is written only by earlier launches: every CTA takes the same branch
	if (done && *done)
		return;

	namespace cgr = cooperative_groups;
	cgr::cluster_group cluster = cgr::this_cluster();
	const int c = (int)cluster.block_rank();
	const bool fuse = (nullptr != dir.st);
	const int it = fuse ? cg_iter(dir.it, dir.st) : 0;

	if (fuse && !dir.start) {	// convergence test of the step just taken

		const double rs = sum_partials_d(dir.rs_part, dir.nrs, red);
		const bool stop = (rs <= dir.st->eps2);

		if ((0 == c) && (0 == threadIdx.x)) {

			dir.st->rs[(it + 1) & 1] = rs;

			if (stop) {

				dir.st->done = 1;
				dir.st->iters = it + 1;
			}
		}

		if (stop)
			return;
	}

	for (int i = threadIdx.x; i < N; i += S::NT)
		tw[i] = twg[i];

	// 1. forward FFT of rows y = c R + seq (the FFT begins with a barrier)
	{
		const int seq = RL::seq();
		const int jt = RL::jt();
		const long y = (long)c * R + seq;
		float2 v[8];
#pragma unroll
		for (int m = 0; m < 8; m++)
			v[m] = r[unwrap_pos(jt + T * m, N, N) + N * y];

		fft_regs<N, RL, false>(v, s, tw);
#pragma unroll
		for (int m = 0; m < 8; m++)
			rowbuf[seq * N + jt + T * m] = v[m];
	}

	cluster.sync();

	// 2. columns cx = c R + seq across the cluster
	{
		const int seq = CLY::seq();
		const int jt = CLY::jt();
		const int cx = c * R + seq;
		float2 v[8], pv[8];
		float2* src[8];
#pragma unroll
		for (int m = 0; m < 8; m++) {

			const int y = unwrap_pos(jt + T * m, N, N);
			src[m] = cluster.map_shared_rank(rowbuf, y / R) + (y % R) * N + cx;
			v[m] = *src[m];
			pv[m] = pinv[cx + (long)(jt + T * m) * N];
		}

		fft_regs<N, CLY, false>(v, s, tw);
#pragma unroll
		for (int m = 0; m < 8; m++)
			v[m] = cmul(v[m], pv[m]);

		fft_regs<N, CLY, true>(v, s, tw);
#pragma unroll
		for (int m = 0; m < 8; m++)
			*src[m] = v[m];
	}

	cluster.sync();

	// 3. inverse FFT of this CTA's rows, uncentred output
	{
		const int seq = RL::seq();
		const int jt = RL::jt();
		const long y = (long)c * R + seq;
		float2 v[8];
#pragma unroll
		for (int m = 0; m < 8; m++)
			v[m] = rowbuf[seq * N + jt + T * m];

		fft_regs<N, RL, true>(v, s, tw);
		double dot = 0.;
#pragma unroll
		for (int m = 0; m < 8; m++) {

			const long i = unwrap_pos(jt + T * m, N, N) + N * y;

			if (!fuse)
				z[i] = v[m];

			if (pdot) {	// Re<pdot, z> (pdot == z: ||z||^2)

				float2 pv = (pdot == z) ? v[m] : pdot[i];
				dot += (double)pv.x * (double)v[m].x + (double)pv.y * (double)v[m].y;
			}
		}

		if (pdot && !fuse) {

			double t = block_sum_d(dot, red);

			if (0 == threadIdx.x)
				dot_part[c] = t;
		}

		if (fuse) {

			float beta = 0.f;

			if (!dir.start) {	// <A p, z> over the cluster, fixed order

				double t = block_sum_d(dot, red);

				if (0 == threadIdx.x)
					cdot = t;

				cluster.sync();
				double dsum = 0.;

				for (int k = 0; k < CL; k++)
					dsum += *cluster.map_shared_rank(&cdot, k);

				cluster.sync();	// no CTA leaves while its cdot is read
				beta = (float)(dsum / dir.st->pap_hist[0]);
			}

			double pr = 0., pp = 0.;
#pragma unroll
			for (int m = 0; m < 8; m++) {

				const long i = unwrap_pos(jt + T * m, N, N) + N * y;
				float2 pn = v[m];

				if (!dir.start) {

					float2 po = dir.p[i];
					pn.x = fmaf(-beta, po.x, pn.x);
					pn.y = fmaf(-beta, po.y, pn.y);
				}

				dir.p[i] = pn;
				float2 rv = dir.r[i];
				pr += (double)pn.x * (double)rv.x + (double)pn.y * (double)rv.y;
				pp += (double)pn.x * (double)pn.x + (double)pn.y * (double)pn.y;
			}

			double t = block_sum_d(pr, red);

			if (0 == threadIdx.x)
				dir.pr_part[c] = t;

			__syncthreads();
			t = block_sum_d(pp, red);

			if (0 == threadIdx.x)
				dir.pp_part[c] = t;
		}
	}
}

} // namespace bn
