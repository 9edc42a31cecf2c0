// Direct non-uniform DFT (the reference's nudft: src/noncart/nudft.c:69-348,
// `bart nufft -s`), evaluated exactly on the GPU:
//   forward  ksp[m, c] = s sum_n img[n, c] exp(i phi_m(n))
//   adjoint  img[n, c] = s sum_m ksp[m, c] exp(-i phi_m(n))
//   phi_m(n) = sum_a 2 pi (-k_a) (n_a - N_a / 2) / N_a
// (linear_phase of the negated trajectory, src/num/filter.c:241-265), with
// s = 1 / sqrt(product of all image dims, coils included), as the reference
// scales it. The phase, in turns of pi, is formed and reduced to [-1, 1] in
// float64, then sincospif gives the factor: accurate for any k and N. Cost is
// M x N x C complex multiply-adds: an oracle-class operator for small sizes.
#pragma once

#include <cuda_runtime.h>

#include "fft_core.cuh"

namespace bn {

enum { NUDFT_THREADS = 256, NUDFT_CHUNK = 256, NUDFT_CC = 8 };

struct NudftGeom {

	int N[3];
	long npix;
	long M;
	long C;
	float scale;
};

// t / pi of the phase; a[a] = -2 k_a / N_a, centre N_a / 2 (float division)
__device__ __forceinline__ float2 nudft_factor(const double a[3], const NudftGeom& g, long n, bool conj)
{
	const int x = (int)(n % g.N[0]);
	const int y = (int)((n / g.N[0]) % g.N[1]);
	const int z = (int)(n / ((long)g.N[0] * g.N[1]));
	double t = a[0] * ((double)x - 0.5 * g.N[0]) + a[1] * ((double)y - 0.5 * g.N[1]) + a[2] * ((double)z - 0.5 * g.N[2]);
	t -= 2. * rint(0.5 * t);
	float s, c;
	sincospif((float)t, &s, &c);
	return make_float2(c, conj ? -s : s);
}

// forward: one thread per sample, pixels staged through shared memory in
// chunks, coils in groups of NUDFT_CC (grid.y)
__global__ void __launch_bounds__(NUDFT_THREADS) k_nudft_fwd(const float4* __restrict__ traj, NudftGeom g,
		const float2* __restrict__ img, float2* __restrict__ ksp)
{
	__shared__ float2 sv[NUDFT_CHUNK][NUDFT_CC];
	const long m = (long)blockIdx.x * blockDim.x + threadIdx.x;
	const int c0 = blockIdx.y * NUDFT_CC;
	const int cn = (int)min((long)NUDFT_CC, g.C - c0);
	double a[3] = { 0., 0., 0. };

	if (m < g.M) {

		float4 k = traj[m];
		a[0] = -2. * (double)k.x / g.N[0];
		a[1] = -2. * (double)k.y / g.N[1];
		a[2] = -2. * (double)k.z / g.N[2];
	}

	float2 acc[NUDFT_CC];
#pragma unroll
	for (int c = 0; c < NUDFT_CC; c++)
		acc[c] = make_float2(0.f, 0.f);

	for (long n0 = 0; n0 < g.npix; n0 += NUDFT_CHUNK) {

		const int nn = (int)min((long)NUDFT_CHUNK, g.npix - n0);
		__syncthreads();

		for (int i = threadIdx.x; i < NUDFT_CHUNK * NUDFT_CC; i += blockDim.x) {

			int j = i / NUDFT_CC;
			int c = i % NUDFT_CC;
			sv[j][c] = ((j < nn) && (c < cn)) ? img[n0 + j + g.npix * (c0 + c)] : make_float2(0.f, 0.f);
		}

		__syncthreads();

		if (m < g.M) {

			for (int j = 0; j < nn; j++) {

				float2 e = nudft_factor(a, g, n0 + j, false);
#pragma unroll
				for (int c = 0; c < NUDFT_CC; c++) {

					float2 v = sv[j][c];
					acc[c].x = fmaf(v.x, e.x, fmaf(-v.y, e.y, acc[c].x));
					acc[c].y = fmaf(v.x, e.y, fmaf(v.y, e.x, acc[c].y));
				}
			}
		}
	}

	if (m < g.M) {
#pragma unroll
		for (int c = 0; c < NUDFT_CC; c++)
			if (c < cn)
				ksp[m + g.M * (c0 + c)] = cscale(acc[c], g.scale);
	}
}

// adjoint: one thread per pixel, samples (phase coefficients and values)
// staged through shared memory in chunks, coils in groups (grid.y)
__global__ void __launch_bounds__(NUDFT_THREADS) k_nudft_adj(const float4* __restrict__ traj, NudftGeom g,
		const float2* __restrict__ ksp, float2* __restrict__ img)
{
	__shared__ double sa[NUDFT_CHUNK][3];
	__shared__ float2 sv[NUDFT_CHUNK][NUDFT_CC];
	const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
	const int c0 = blockIdx.y * NUDFT_CC;
	const int cn = (int)min((long)NUDFT_CC, g.C - c0);

	float2 acc[NUDFT_CC];
#pragma unroll
	for (int c = 0; c < NUDFT_CC; c++)
		acc[c] = make_float2(0.f, 0.f);

	for (long m0 = 0; m0 < g.M; m0 += NUDFT_CHUNK) {

		const int mm = (int)min((long)NUDFT_CHUNK, g.M - m0);
		__syncthreads();

		for (int j = threadIdx.x; j < NUDFT_CHUNK; j += blockDim.x) {

			float4 k = (j < mm) ? traj[m0 + j] : make_float4(0.f, 0.f, 0.f, 0.f);
			sa[j][0] = -2. * (double)k.x / g.N[0];
			sa[j][1] = -2. * (double)k.y / g.N[1];
			sa[j][2] = -2. * (double)k.z / g.N[2];
		}

		for (int i = threadIdx.x; i < NUDFT_CHUNK * NUDFT_CC; i += blockDim.x) {

			int j = i / NUDFT_CC;
			int c = i % NUDFT_CC;
			sv[j][c] = ((j < mm) && (c < cn)) ? ksp[m0 + j + g.M * (c0 + c)] : make_float2(0.f, 0.f);
		}

		__syncthreads();

		if (n < g.npix) {

			for (int j = 0; j < mm; j++) {

				double a[3] = { sa[j][0], sa[j][1], sa[j][2] };
				float2 e = nudft_factor(a, g, n, true);
#pragma unroll
				for (int c = 0; c < NUDFT_CC; c++) {

					float2 v = sv[j][c];
					acc[c].x = fmaf(v.x, e.x, fmaf(-v.y, e.y, acc[c].x));
					acc[c].y = fmaf(v.x, e.y, fmaf(v.y, e.x, acc[c].y));
				}
			}
		}
	}

	if (n < g.npix) {
#pragma unroll
		for (int c = 0; c < NUDFT_CC; c++)
			if (c < cn)
				img[n + g.npix * (c0 + c)] = cscale(acc[c], g.scale);
	}
}

} // namespace bn
