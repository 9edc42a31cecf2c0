// NUFFT device kernels: fused FFT passes over the 2x oversampled grid and
// Kaiser-Bessel gridding / degridding.
//
// Grid convention. For an image axis of N pixels the oversampled axis has
// L = 2N cells stored in DFT order: cell j' holds the image's Fourier
// transform at frequency j'/2 (j' < N) or (j' - 2N)/2 (j' >= N), in cycles
// per FOV. Image pixel n enters the length-L transform at position
// (n - N/2) mod L (zero elsewhere), which is the reference's centred
// transform (fftmod / linphase chain, src/noncart/nufft.c:196-248, 1410-1423)
// written as an index map instead of phase multiplies. The reference's
// sub-grid s, tap w (src/noncart/nufft.c:158-188) is centred cell
// j = 2w + s, i.e. DFT cell (j + N) mod L.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_core.cuh"

namespace bn {

enum { KB_TABLE_N = 1000 };	// kb_size_max, src/noncart/grid.c:38

// Element layouts ------------------------------------------------------------

// smem element stride for B sequences: odd, so 8-byte accesses of a
// half-warp land in distinct banks
__host__ __device__ __forceinline__ int smem_stride(int B) { return B | 1; }

// position of input element n (of n_in) inside the length-L transform
__device__ __forceinline__ int wrap_pos(int n, int n_in, int L)
{
	int p = n - n_in / 2;
	return (p < 0) ? p + L : p;
}

// inverse of wrap_pos: which input element sits at position p (>= n_in: none)
__device__ __forceinline__ int unwrap_pos(int p, int n_in, int L)
{
	int n = p + n_in / 2;
	return (n >= L) ? n - L : n;
}

// Row pass, forward ----------------------------------------------------------
//
// Rows r in [0, R): yz = r % YZ, c = r / YZ. Input row x in [0, X):
//   v = img[x + X*yz (+ X*YZ*c unless maps)] (* maps[x + X*yz + X*YZ*c])
//       * ax[x] * ayz[yz]                          (apodisation, optional)
// placed at wrap_pos(x, X, L), transformed, written to out[p + L*r].
// One block: B rows, B*L/8 threads.
template <int L>
__global__ void __launch_bounds__(1024) k_rows_fwd(const float2* __restrict__ img, const float2* __restrict__ maps,
		const float* __restrict__ ax, const float* __restrict__ ayz,
		int X, long YZ, long R, int B, float2* __restrict__ out, const float2* __restrict__ twg)
{
	extern __shared__ float2 smem[];
	const int SB = smem_stride(B);
	float2* s = smem;
	float2* tw = smem + L * SB;

	for (int i = threadIdx.x; i < L; i += blockDim.x)
		tw[i] = twg[i];

	const long r0 = (long)blockIdx.x * B;

	for (int e = threadIdx.x; e < L * B; e += blockDim.x) {

		int b = e / L;
		int p = e - b * L;
		long r = r0 + b;
		int n = unwrap_pos(p, X, L);
		float2 v = make_float2(0.f, 0.f);

		if ((n < X) && (r < R)) {

			long yz = r % YZ;
			long c = r / YZ;

			if (maps) {

				v = cmul(img[n + X * yz], maps[n + X * yz + X * YZ * c]);

			} else {

				v = img[n + X * yz + X * YZ * c];
			}

			if (ax)
				v = cscale(v, ax[n] * ayz[yz]);
		}

		s[p * SB + b] = v;
	}

	__syncthreads();

	fft_block<L, false>(s, SB, B, tw);

	for (int e = threadIdx.x; e < L * B; e += blockDim.x) {

		int b = e / L;
		int p = e - b * L;
		long r = r0 + b;

		if (r < R)
			out[p + (long)L * r] = s[p * SB + b];
	}
}

// Column pass ------------------------------------------------------------------
//
// Sequences (cx, o): cx in [0, W) contiguous columns, o in [0, O) outer index.
// Input element n of sequence (cx, o) is in[cx + n*ies + o*ios] for n < n_in,
// placed at wrap_pos(n, n_in, L) when wrap_in, else at n.
// MODE 0: forward FFT; 1: inverse FFT; 2: forward, * psf, inverse (Toeplitz).
// Output element n' < n_out is taken from position wrap_pos(n', n_out, L)
// when wrap_out, else n', and written to out[cx + n'*oes + o*oos].
// psf element for position p: psf[cx + p*pes + (o % pmod)*pos].
// One block: B columns of one outer index, B*L/8 threads; grid (ceil(W/B), O).
template <int L, int MODE>
__global__ void __launch_bounds__(1024) k_cols(const float2* __restrict__ in, long ies, long ios, int n_in, int wrap_in,
		float2* __restrict__ out, long oes, long oos, int n_out, int wrap_out,
		int W, int B, const float2* __restrict__ psf, long pes, long pmod, long pos,
		const float2* __restrict__ twg)
{
	extern __shared__ float2 smem[];
	const int SB = smem_stride(B);
	float2* s = smem;
	float2* tw = smem + L * SB;

	for (int i = threadIdx.x; i < L; i += blockDim.x)
		tw[i] = twg[i];

	const int cx0 = blockIdx.x * B;
	const long o = blockIdx.y;
	const float2* inp = in + o * ios + cx0;

	for (int e = threadIdx.x; e < L * B; e += blockDim.x) {

		int p = e / B;
		int b = e - p * B;
		int n = wrap_in ? unwrap_pos(p, n_in, L) : p;
		float2 v = make_float2(0.f, 0.f);

		if ((n < n_in) && (cx0 + b < W))
			v = inp[b + n * ies];

		s[p * SB + b] = v;
	}

	__syncthreads();

	if constexpr (MODE == 1) {

		fft_block<L, true>(s, SB, B, tw);

	} else {

		fft_block<L, false>(s, SB, B, tw);
	}

	if constexpr (MODE == 2) {

		const float2* pp = psf + (o % pmod) * pos + cx0;

		for (int e = threadIdx.x; e < L * B; e += blockDim.x) {

			int p = e / B;
			int b = e - p * B;

			if (cx0 + b < W)
				s[p * SB + b] = cmul(s[p * SB + b], pp[b + p * pes]);
		}

		__syncthreads();

		fft_block<L, true>(s, SB, B, tw);
	}

	float2* outp = out + o * oos + cx0;

	for (int e = threadIdx.x; e < n_out * B; e += blockDim.x) {

		int n = e / B;
		int b = e - n * B;
		int p = wrap_out ? wrap_pos(n, n_out, L) : n;

		if (cx0 + b < W)
			outp[b + n * oes] = s[p * SB + b];
	}
}

// Row pass, inverse --------------------------------------------------------------
//
// Input rows in[p + L*(yz + YZ*c)], p < L. Each block takes B consecutive yz
// rows and coils [c0, c1): inverse FFT per row, keep x < X from
// wrap_pos(x, X, L), scale by ax[x]*ayz[yz] (optional) and either
//   maps != 0: accumulate sum_c conj(maps[x + X*yz + X*YZ*c]) * row
//              into out[x + X*yz + X*YZ*g] (g = blockIdx.y, partial per group)
//   maps == 0: write out[x + X*yz + X*YZ*c] per coil.
// grid (ceil(YZ/B), groups); coils per group cpg.
template <int L>
__global__ void __launch_bounds__(1024) k_rows_inv(const float2* __restrict__ in, const float2* __restrict__ maps,
		const float* __restrict__ ax, const float* __restrict__ ayz,
		int X, long YZ, int C, int cpg, int B, float2* __restrict__ out, const float2* __restrict__ twg)
{
	extern __shared__ float2 smem[];
	const int SB = smem_stride(B);
	float2* s = smem;
	float2* tw = smem + L * SB;

	for (int i = threadIdx.x; i < L; i += blockDim.x)
		tw[i] = twg[i];

	const long yz0 = (long)blockIdx.x * B;
	const int g = blockIdx.y;
	const int c0 = g * cpg;
	const int c1 = min(C, c0 + cpg);

	// each thread owns up to OWN output elements (x, b) across the coil loop
	constexpr int OWN = 8;
	float2 acc[OWN];
#pragma unroll
	for (int k = 0; k < OWN; k++)
		acc[k] = make_float2(0.f, 0.f);

	for (int c = c0; c < c1; c++) {

		for (int e = threadIdx.x; e < L * B; e += blockDim.x) {

			int b = e / L;
			int p = e - b * L;
			long yz = yz0 + b;
			float2 v = make_float2(0.f, 0.f);

			if (yz < YZ)
				v = in[p + (long)L * (yz + YZ * c)];

			s[p * SB + b] = v;
		}

		__syncthreads();

		fft_block<L, true>(s, SB, B, tw);

#pragma unroll
		for (int k = 0; k < OWN; k++) {

			int e = threadIdx.x + k * blockDim.x;

			if (e >= X * B)
				break;

			int b = e / X;
			int x = e - b * X;
			long yz = yz0 + b;

			if (yz >= YZ)
				continue;

			float2 v = s[wrap_pos(x, X, L) * SB + b];

			if (ax)
				v = cscale(v, ax[x] * ayz[yz]);

			if (maps) {

				float2 m = maps[x + X * yz + X * YZ * c];
				acc[k] = cadd(acc[k], cmulc(v, m));

			} else {

				out[x + X * yz + X * YZ * c] = v;
			}
		}

		__syncthreads();
	}

	if (maps) {
#pragma unroll
		for (int k = 0; k < OWN; k++) {

			int e = threadIdx.x + k * blockDim.x;

			if (e >= X * B)
				break;

			int b = e / X;
			int x = e - b * X;
			long yz = yz0 + b;

			if (yz < YZ)
				out[x + X * yz + X * YZ * g] = acc[k];
		}
	}
}

// Kaiser-Bessel taps ----------------------------------------------------------------

// intlookup (src/noncart/grid.c:120-149): x *= 2; idx = (int)(x*(n-1));
// lerp in float64 ((1. - c) * a + c * b), rounded to float. Explicit
// round-to-nearest intrinsics keep the compiler from contracting into FMAs,
// so the result is bit-identical to the reference's.
__device__ __forceinline__ float kb_lookup(const float* kb, float x)
{
	x = __fmul_rn(x, 2.0f);
	float xs = __fmul_rn(x, (float)(KB_TABLE_N - 1));
	int idx = (int)xs;
	float fpart = __fsub_rn(xs, (float)idx);
	double a = (double)kb[idx];
	double b = (double)kb[idx + 1];
	double c = (double)fpart;
	double r = __dadd_rn(__dmul_rn(__dsub_rn(1.0, c), a), __dmul_rn(c, b));
	return __double2float_rn(r);
}

enum { MAX_AXIS_TAPS = 10 };

struct AxisTaps {

	int n;
	int cell[MAX_AXIS_TAPS];	// DFT-order cell on the 2N axis
	float w[MAX_AXIS_TAPS];
};

// Taps of one axis for both sub-grid shifts (grid2H_decomp / grid_point_gen,
// src/noncart/nufft.c:158-188, src/noncart/grid.c:403-465):
//   pos_s = float(k + (-s/2)) + float(N/2)   (width hw = w/2 on the N-grid)
//   taps t = ceil(pos_s - hw/2) .. floor(pos_s + hw/2)  (float64 bounds)
//   weight = intlookup(|t - pos_s| / hw)
//   cell: centred j = 2 t + s  ->  DFT order (j + N) mod 2N
// Non-periodic: taps clipped to [0, N-1]; periodic: t mod N.
__device__ __forceinline__ void axis_taps(float k, int N, float hw, int periodic, const float* kb, AxisTaps& t)
{
	t.n = 0;

	if (1 == N) {	// singleton axis: one tap at 0 with intlookup(0)

		t.cell[0] = 0;
		t.w[0] = kb_lookup(kb, 0.f);
		t.n = 1;
		return;
	}

	const int L = 2 * N;
	const float half = (float)(N / 2);
	const double h2 = 0.5 * (double)hw;

#pragma unroll
	for (int s = 0; s < 2; s++) {

		float pos = __fadd_rn(__fadd_rn(k, s ? -0.5f : -0.0f), half);
		int sti = (int)ceil((double)pos - h2);
		int eni = (int)floor((double)pos + h2);

		if (!periodic) {

			sti = max(sti, 0);
			eni = min(eni, N - 1);
		}

		for (int w = sti; (w <= eni) && (t.n < MAX_AXIS_TAPS); w++) {

			float frac = fabsf(__fsub_rn((float)w, pos));
			float val = kb_lookup(kb, __fdiv_rn(frac, hw));
			int wm = periodic ? (((w % N) + N) % N) : w;
			int j = 2 * wm + s + N;

			if (j >= L)
				j -= L;

			t.cell[t.n] = j;
			t.w[t.n] = val;
			t.n++;
		}
	}
}

struct GridGeom {

	int N[3];	// image size per axis
	int G[3];	// grid size per axis (2N, or 1)
	long gsz;	// cells per channel
	float hw;	// kernel width on the N-grid (conf.width / 2)
	int periodic;
};

// Degridding (forward interpolation), one thread per sample, coils
// [blockIdx.y*cpc, ...). ksp[m + M*c] = sum_taps w * grid[cell + gsz*c].
// The combined weight is ((1*wz)*wy)*wx in float32 as in grid_point_gen.
__global__ void k_degrid(const float4* __restrict__ traj, long M, GridGeom g, int C, int cpc,
		const float2* __restrict__ grid, float2* __restrict__ ksp, const float* __restrict__ kbg)
{
	__shared__ float kb[KB_TABLE_N + 1];

	for (int i = threadIdx.x; i <= KB_TABLE_N; i += blockDim.x)
		kb[i] = kbg[i];

	__syncthreads();

	long m = (long)blockIdx.x * blockDim.x + threadIdx.x;

	if (m >= M)
		return;

	float4 k = traj[m];
	AxisTaps tx, ty, tz;
	axis_taps(k.x, g.N[0], g.hw, g.periodic, kb, tx);
	axis_taps(k.y, g.N[1], g.hw, g.periodic, kb, ty);
	axis_taps(k.z, g.N[2], g.hw, g.periodic, kb, tz);

	const int c0 = blockIdx.y * cpc;
	const int c1 = min(C, c0 + cpc);

	for (int c = c0; c < c1; c++) {

		const float2* gc = grid + g.gsz * c;
		float2 acc = make_float2(0.f, 0.f);

		for (int a = 0; a < tz.n; a++) {

			float dz = tz.w[a];
			long oz = (long)tz.cell[a] * g.G[1];

			for (int bb = 0; bb < ty.n; bb++) {

				float dzy = __fmul_rn(dz, ty.w[bb]);
				long oy = (oz + ty.cell[bb]) * g.G[0];

				for (int cc = 0; cc < tx.n; cc++) {

					float d = __fmul_rn(dzy, tx.w[cc]);
					float2 v = gc[oy + tx.cell[cc]];
					acc.x = fmaf(v.x, d, acc.x);
					acc.y = fmaf(v.y, d, acc.y);
				}
			}
		}

		ksp[m + M * c] = acc;
	}
}

// Gridding (adjoint spreading) with float2 atomics into the grid (must be
// zeroed). One thread per sample, coils as in k_degrid.
__global__ void k_grid_atomic(const float4* __restrict__ traj, long M, GridGeom g, int C, int cpc,
		const float2* __restrict__ ksp, float2* __restrict__ grid, const float* __restrict__ kbg)
{
	__shared__ float kb[KB_TABLE_N + 1];

	for (int i = threadIdx.x; i <= KB_TABLE_N; i += blockDim.x)
		kb[i] = kbg[i];

	__syncthreads();

	long m = (long)blockIdx.x * blockDim.x + threadIdx.x;

	if (m >= M)
		return;

	float4 k = traj[m];
	AxisTaps tx, ty, tz;
	axis_taps(k.x, g.N[0], g.hw, g.periodic, kb, tx);
	axis_taps(k.y, g.N[1], g.hw, g.periodic, kb, ty);
	axis_taps(k.z, g.N[2], g.hw, g.periodic, kb, tz);

	const int c0 = blockIdx.y * cpc;
	const int c1 = min(C, c0 + cpc);

	for (int c = c0; c < c1; c++) {

		float2 val = ksp[m + M * c];

		if ((0.f == val.x) && (0.f == val.y))
			continue;	// grid(): samples that are zero in all channels are skipped

		float2* gc = grid + g.gsz * c;

		for (int a = 0; a < tz.n; a++) {

			float dz = tz.w[a];
			long oz = (long)tz.cell[a] * g.G[1];

			for (int bb = 0; bb < ty.n; bb++) {

				float dzy = __fmul_rn(dz, ty.w[bb]);
				long oy = (oz + ty.cell[bb]) * g.G[0];

				for (int cc = 0; cc < tx.n; cc++) {

					float d = __fmul_rn(dzy, tx.w[cc]);
					atomicAdd(&gc[oy + tx.cell[cc]], make_float2(val.x * d, val.y * d));
				}
			}
		}
	}
}

} // namespace bn
