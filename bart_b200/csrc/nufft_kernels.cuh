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
#include "fft512.cuh"

namespace bn {

enum { KB_TABLE_N = 1000 };	// kb_size_max, src/noncart/grid.c:38

// A DFT of logical length n run on the power-of-two FFT of the kernel's
// template length L. n == L: the FFT itself. n < L (any n with 2n - 1 <= L):
// Bluestein's chirp-z algorithm (IEEE Trans. Audio Electroacoust. 18(4),
// 1970): with c_j = exp(-i pi j^2 / n), the forward DFT is
//   X_k = c_k sum_j (x_j c_j) conj(c_{k-j}),
// a linear convolution computed as a length-L circular one:
//   X = c . IFFT_L(FFT_L(c . x) . bf),  bf = FFT_L(conj(c) wrapped) / L,
// and the inverse DFT the same with conj(c) and bi = FFT_L(c wrapped) / L.
// Positions j >= n hold zeros before and after.
struct Dft {

	int n;			// logical length
	const float2* chirp;	// [n] c_j (Bluestein only)
	const float2* bf;	// [L] forward filter spectrum / L
	const float2* bi;	// [L] inverse filter spectrum / L
};

// DFT of the register set v (positions reg_pos(m), see fft_regs); for
// Bluestein the caller has loaded zeros at positions >= d.n and gets zeros
// there back. Same barrier contract as fft_regs.
template <int L, typename LAY, bool INV, bool BLUE>
__device__ __forceinline__ void dft_regs(float2 (&v)[8], float2* s, const float2* tw, const Dft& d,
		bool half_in = false)
{
	if constexpr (!BLUE) {

		fft_regs<L, LAY, INV>(v, s, tw, half_in);
		return;
	}

#pragma unroll
	for (int m = 0; m < 8; m++) {

		int p = reg_pos<L, LAY>(m);
		float2 c = (p < d.n) ? d.chirp[p] : make_float2(0.f, 0.f);
		v[m] = INV ? cmulc(v[m], c) : cmul(v[m], c);
	}

	fft_regs<L, LAY, false>(v, s, tw);
	const float2* b = INV ? d.bi : d.bf;
#pragma unroll
	for (int m = 0; m < 8; m++)
		v[m] = cmul(v[m], b[reg_pos<L, LAY>(m)]);

	fft_regs<L, LAY, true>(v, s, tw);
#pragma unroll
	for (int m = 0; m < 8; m++) {

		int p = reg_pos<L, LAY>(m);
		float2 c = (p < d.n) ? d.chirp[p] : make_float2(0.f, 0.f);
		v[m] = INV ? cmulc(v[m], c) : cmul(v[m], c);
	}
}

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

// float64 block reduction; the result is valid in thread 0. blockDim.x must be
// a multiple of 32.
__device__ __forceinline__ double block_sum_d(double v, double* sh)
{
	for (int o = 16; o > 0; o >>= 1)
		v += __shfl_down_sync(0xffffffffu, v, o);

	__syncthreads();

	if (0 == threadIdx.x % 32)
		sh[threadIdx.x / 32] = v;

	__syncthreads();

	double r = 0.;

	if (threadIdx.x < 32) {

		r = (threadIdx.x < blockDim.x / 32) ? sh[threadIdx.x] : 0.;

		for (int o = 16; o > 0; o >>= 1)
			r += __shfl_down_sync(0xffffffffu, r, o);
	}

	return r;
}

// fixed-order sum of n float64 partials, the same value in every thread
__device__ __forceinline__ double sum_partials_d(const double* part, int n, double* sh)
{
	double v = 0.;

	for (int i = threadIdx.x; i < n; i += blockDim.x)
		v += part[i];

	double r = block_sum_d(v, sh);

	if (0 == threadIdx.x)
		sh[0] = r;

	__syncthreads();
	r = sh[0];
	__syncthreads();
	return r;
}

// flexible CG: largest truncation (directions kept) and ring size
enum { FCG_MAX_M = 16, FCG_RING = FCG_MAX_M + 1 };

// device-side state of the CG solve
struct CgScalars {

	double rs[2];		// ||r||^2 of iteration it in rs[it & 1]
	double eps2;		// stop when ||r||^2 <= eps2
	double b2;		// ||A^H y||^2
	int done;		// set once converged (or p^H A p == 0)
	int iters;		// iterations completed
	int it;			// iteration being run (device-driven loop)
	int maxiter;		// iteration limit of the current solve
	double pap_hist[FCG_RING];	// <p_j, (A^H A + lambda) p_j>, slot j % FCG_RING (flexible CG)
	double best_rs;		// smallest ||r||^2 so far (flexible CG stall test)
	double best_hist[4];	// best_rs after iteration j, slot j % 4
	int best_it;		// iteration count at best_rs
	int net_off;		// learned preconditioner switched off (stall fallback)
	int restart_it;		// flexible CG direction history starts here
	int net_iters;		// learned preconditioner used in iterations < net_iters (0: no limit)
	float rnorm;		// ||r|| of the current residual
	float rinv;		// 1 / ||r|| (0 for r = 0)
	float scale;		// data scaling used
	float inv_scale;	// float(1 / scale)
	int f32;		// plain CG keeps ||r||^2, p^H A p, alpha and beta in float32
};

// iteration index of a CG pass: the host's, or the device counter when the
// loop runs inside a graph (it < 0)
__device__ __forceinline__ int cg_iter(int it, const CgScalars* st) { return (it < 0) ? st->it : it; }

// Plain-CG scalars in the reference's precision when st->f32 is set:
// conjgrad (src/iter/italgos.c:518-554) sums its dot products in float64
// but stores rsold, rsnew, pAp, alpha and beta as float, and divides in
// float. cg_keep rounds a float64 sum as the reference stores it; cg_ratio
// is alpha = rsold / pAp or beta = rsnew / rsold.
__device__ __forceinline__ double cg_keep(const CgScalars* st, double v)
{
	return st->f32 ? (double)(float)v : v;
}

__device__ __forceinline__ float cg_ratio(const CgScalars* st, double num, double den)
{
	return st->f32 ? __fdiv_rn((float)num, (float)den) : (float)(num / den);
}

// three fixed-order float64 sums of partials in one block reduction, the
// same values in every thread (sh: 3 doubles per warp)
__device__ __forceinline__ double3 sum_partials3_d(const double* a, int na, const double* b, int nb,
		const double* c, int nc, double* sh)
{
	double3 v = make_double3(0., 0., 0.);
	const int n = max(na, max(nb, nc));

	for (int i = threadIdx.x; i < n; i += blockDim.x) {

		if (i < na)
			v.x += a[i];

		if (i < nb)
			v.y += b[i];

		if (i < nc)
			v.z += c[i];
	}

	for (int o = 16; o > 0; o >>= 1) {

		v.x += __shfl_down_sync(0xffffffffu, v.x, o);
		v.y += __shfl_down_sync(0xffffffffu, v.y, o);
		v.z += __shfl_down_sync(0xffffffffu, v.z, o);
	}

	__syncthreads();

	if (0 == threadIdx.x % 32) {

		sh[3 * (threadIdx.x / 32) + 0] = v.x;
		sh[3 * (threadIdx.x / 32) + 1] = v.y;
		sh[3 * (threadIdx.x / 32) + 2] = v.z;
	}

	__syncthreads();
	double3 r = make_double3(0., 0., 0.);

	for (int w = 0; w < (int)(blockDim.x / 32); w++) {

		r.x += sh[3 * w + 0];
		r.y += sh[3 * w + 1];
		r.z += sh[3 * w + 2];
	}

	__syncthreads();
	return r;
}

// Row pass, forward, first step of a CG iteration (conjgrad,
// src/iter/italgos.c:538-566, reordered so that the direction update of the
// previous iteration happens while loading):
//   it == 0: p = b;  else: rs = ||r||^2 (from the update's partials),
//   stop if rs <= eps2, beta = rs / rs_prev, p = r + beta p_prev.
// p_prev and p_cur are distinct buffers (blocks of other coils still read
// p_prev while coil 0 writes p_cur); the CG step copies p_cur back to p_prev.
// Rows of coil 0 write p and the partial ||p||^2 (for lambda ||p||^2 in
// p^H (A^H A + lambda) p); every row multiplies by its coil's map and runs the
// forward transform like k_rows_fwd.
template <int L, int B, bool BLUE>
__global__ void __launch_bounds__(B * L / 8, (1024 / (B * L / 8)) > 0 ? 1024 / (B * L / 8) : 1) k_rows_fwd_cg(const float2* __restrict__ bvec, const float2* __restrict__ r,
		const float2* __restrict__ p_prev, float2* __restrict__ p_cur, const float2* __restrict__ maps,
		const float* __restrict__ ax, const float* __restrict__ ayz,
		int X, long YZ, long R, float2* __restrict__ out, const float2* __restrict__ twg,
		CgScalars* st, int it, const double* __restrict__ rs_part, int nrs, double* __restrict__ pp_part, Dft d)
{
	using LAY = RowLayout<L, B>;
	const int dn = BLUE ? d.n : L;	// logical DFT length (compile-time for the FFT itself)
	constexpr int NT = B * L / 8;
	extern __shared__ float2 smem[];
	__shared__ double red[32];
	float2* s = smem;
	float2* tw = smem + LAY::SMEM;

	if (st->done)
		return;

	it = cg_iter(it, st);
	float beta = 0.f;

	if (it > 0) {

		double rs = cg_keep(st, sum_partials_d(rs_part, nrs, red));
		double rs_prev = st->rs[(it - 1) & 1];
		bool stop = (rs <= st->eps2);

		if (0 == blockIdx.x && 0 == threadIdx.x) {

			st->rs[it & 1] = rs;

			if (stop) {

				st->done = 1;
				st->iters = it;
			}
		}

		if (stop)
			return;

		beta = cg_ratio(st, rs, rs_prev);
	}

	for (int i = threadIdx.x; i < L; i += NT)
		tw[i] = twg[i];

	const long row = (long)blockIdx.x * B + LAY::seq();
	const bool valid = (row < R);
	const long yz = valid ? row % YZ : 0;
	const long c = valid ? row / YZ : 0;
	double pp = 0.;
	float2 v[8];

#pragma unroll
	for (int m = 0; m < 8; m++) {

		int p = reg_pos<L, LAY>(m);
		int n = (p < dn) ? unwrap_pos(p, X, dn) : X;
		v[m] = make_float2(0.f, 0.f);

		if (valid && (n < X)) {

			long i = n + X * yz;
			float2 pv;

			if (0 == it) {

				pv = bvec[i];

			} else {

				float2 rv = r[i];
				float2 po = p_prev[i];
				pv.x = fmaf(beta, po.x, rv.x);
				pv.y = fmaf(beta, po.y, rv.y);
			}

			if (0 == c) {

				p_cur[i] = pv;
				pp += (double)pv.x * (double)pv.x + (double)pv.y * (double)pv.y;
			}

			float2 w = cmul(pv, maps[i + X * YZ * c]);
			v[m] = ax ? cscale(w, ax[n] * ayz[yz]) : w;
		}
	}

	double t = block_sum_d(pp, red);

	if (0 == threadIdx.x)
		pp_part[blockIdx.x] = t;

	dft_regs<L, LAY, false, BLUE>(v, s, tw, d, 2 * X == L);

	if (valid) {
#pragma unroll
		for (int m = 0; m < 8; m++) {

			int p = reg_pos<L, LAY>(m);

			if (p < dn)
				out[p + (long)dn * row] = v[m];
		}
	}
}

// Row pass, forward ----------------------------------------------------------
//
// Rows r in [0, R): yz = r % YZ, c = r / YZ. Input row x in [0, X):
//   v = img[x + X*yz (+ X*YZ*c unless maps)] (* maps[x + X*yz + X*YZ*c])
//       * ax[x] * ayz[yz]                          (apodisation, optional)
// placed at wrap_pos(x, X, L), transformed, written to out[p + L*r].
// One block: B rows, B*L/8 threads; a warp reads and writes consecutive
// elements of one row straight from / into the FFT's registers.
template <int L, int B, bool BLUE>
__global__ void __launch_bounds__(B * L / 8, (1024 / (B * L / 8)) > 0 ? 1024 / (B * L / 8) : 1) k_rows_fwd(const float2* __restrict__ img, const float2* __restrict__ maps,
		const float* __restrict__ ax, const float* __restrict__ ayz,
		int X, long YZ, long R, float2* __restrict__ out, const float2* __restrict__ twg, const int* done, Dft d)
{
	using LAY = RowLayout<L, B>;
	const int dn = BLUE ? d.n : L;	// logical DFT length (compile-time for the FFT itself)
	constexpr int NT = B * L / 8;
	extern __shared__ float2 smem[];
	float2* s = smem;
	float2* tw = smem + LAY::SMEM;

	if (done && *done)
		return;

	for (int i = threadIdx.x; i < L; i += NT)
		tw[i] = twg[i];

	const long row = (long)blockIdx.x * B + LAY::seq();
	const bool valid = (row < R);
	const long yz = valid ? row % YZ : 0;
	const long c = valid ? row / YZ : 0;
	float2 v[8];

#pragma unroll
	for (int m = 0; m < 8; m++) {

		int p = reg_pos<L, LAY>(m);
		int n = (p < dn) ? unwrap_pos(p, X, dn) : X;
		v[m] = make_float2(0.f, 0.f);

		if (valid && (n < X)) {

			float2 w = maps ? cmul(img[n + X * yz], maps[n + X * yz + X * YZ * c])
					: img[n + X * yz + X * YZ * c];
			v[m] = ax ? cscale(w, ax[n] * ayz[yz]) : w;
		}
	}

	dft_regs<L, LAY, false, BLUE>(v, s, tw, d, 2 * X == L);

	if (valid) {
#pragma unroll
		for (int m = 0; m < 8; m++) {

			int p = reg_pos<L, LAY>(m);

			if (p < dn)
				out[p + (long)dn * row] = v[m];
		}
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
// Global loads go straight into the first FFT stage's registers and results
// leave from the last stage's registers (B consecutive columns per access).
// the Toeplitz column pass of three-stage power-of-two lengths keeps two
// exchange buffers when they fit (fft_regs_db)
__host__ __device__ constexpr bool cols_double_buffered(int MODE, bool BLUE, int L, int B)
{
	return (2 == MODE) && !BLUE && (L >= 128) && (L <= 512)
		&& ((2 * L * (B | 1) + L) * 8 <= 200 * 1024);
}

template <int L, int B, int MODE, bool BLUE>
__global__ void __launch_bounds__(B * L / 8, (1024 / (B * L / 8)) > 0 ? 1024 / (B * L / 8) : 1) k_cols(const float2* __restrict__ in, long ies, long ios, int n_in, int wrap_in,
		float2* __restrict__ out, long oes, long oos, int n_out, int wrap_out,
		int W, const float2* __restrict__ psf, long pes, long pmod, long pos,
		const float2* __restrict__ twg, const int* done, Dft d)
{
	using LAY = ColLayout<L, B>;
	const int dn = BLUE ? d.n : L;	// logical DFT length (compile-time for the FFT itself)
	constexpr int NT = B * L / 8;
	constexpr bool DB = cols_double_buffered(MODE, BLUE, L, B);
	extern __shared__ float2 smem[];
	float2* s = smem;
	float2* tw = smem + (DB ? 2 : 1) * LAY::SMEM;

	if (done && *done)
		return;

	for (int i = threadIdx.x; i < L; i += NT)
		tw[i] = twg[i];

	const int cx = blockIdx.x * B + LAY::seq();
	const bool valid = (cx < W);
	const long o = blockIdx.y;
	const float2* inp = in + o * ios + cx;

	float2 v[8];
#pragma unroll
	for (int m = 0; m < 8; m++) {

		int p = reg_pos<L, LAY>(m);
		int n = (p >= dn) ? n_in : (wrap_in ? unwrap_pos(p, n_in, dn) : p);
		v[m] = (valid && (n < n_in)) ? inp[n * ies] : make_float2(0.f, 0.f);
	}

	if constexpr (DB) {	// Toeplitz with double-buffered exchanges; the PSF column loads first

		const float2* pp = psf + (o % pmod) * pos + cx;
		float2 pv[8];
#pragma unroll
		for (int m = 0; m < 8; m++)
			pv[m] = valid ? pp[reg_pos<L, LAY>(m) * pes] : make_float2(0.f, 0.f);

		fft_regs_db<L, LAY, false>(v, s, s + LAY::SMEM, tw, wrap_in && (2 * n_in == L));
#pragma unroll
		for (int m = 0; m < 8; m++)
			v[m] = cmul(v[m], pv[m]);

		fft_regs_db<L, LAY, true>(v, s, s + LAY::SMEM, tw);

	} else if constexpr (MODE == 1) {	// the twiddle table must be complete before the first stage reads it

		dft_regs<L, LAY, true, BLUE>(v, s, tw, d);

	} else {

		dft_regs<L, LAY, false, BLUE>(v, s, tw, d, wrap_in && (2 * n_in == L));
	}

	if constexpr ((MODE == 2) && !DB) {

		const float2* pp = psf + (o % pmod) * pos + cx;
#pragma unroll
		for (int m = 0; m < 8; m++) {

			int p = reg_pos<L, LAY>(m);

			if (valid && (p < dn))
				v[m] = cmul(v[m], pp[p * pes]);
		}

		dft_regs<L, LAY, true, BLUE>(v, s, tw, d);
	}

	float2* outp = out + o * oos + cx;

	if (valid) {
#pragma unroll
		for (int m = 0; m < 8; m++) {

			int p = reg_pos<L, LAY>(m);
			int n = (p >= dn) ? n_out : (wrap_out ? unwrap_pos(p, n_out, dn) : p);

			if (n < n_out)
				outp[n * oes] = v[m];
		}
	}
}

// Toeplitz column pass for 512-point columns in two-stage transforms
// (fft512_regs): sixteen columns per block, sixteen threads per column, 32
// elements per thread. The same positions, PSF product and crop as k_cols
// MODE 2; one shared-memory exchange and one barrier per transform, plus the
// barrier for the twiddle table and the one between the two transforms.
enum { TOE512_B = 16 };

__global__ void __launch_bounds__(TOE512_B * 16, 2) k_cols_toe512(const float2* __restrict__ in, long ies, long ios,
		int n_in, int wrap_in, float2* __restrict__ out, long oes, long oos, int n_out, int wrap_out,
		int W, const float2* __restrict__ psf, long pes, long pmod, long pos,
		const float2* __restrict__ twg, const int* done)
{
	constexpr int L = 512, SB = TOE512_B;
	extern __shared__ float2 smem[];
	float2* s = smem;
	float2* tw = smem + L * SB;

	if (done && *done)
		return;

	for (int i = threadIdx.x; i < L; i += blockDim.x)
		tw[i] = twg[i];

	const int b = threadIdx.x % TOE512_B, t = threadIdx.x / TOE512_B;
	const int cx = blockIdx.x * TOE512_B + b;
	const bool valid = (cx < W);
	const long o = blockIdx.y;
	const float2* inp = in + o * ios + cx;

	float2 v[32];
#pragma unroll
	for (int m = 0; m < 32; m++) {

		const int p = t + 16 * m;
		const int n = wrap_in ? unwrap_pos(p, n_in, L) : p;
		v[m] = (valid && (n < n_in)) ? inp[n * ies] : make_float2(0.f, 0.f);
	}

	__syncthreads();	// the twiddle table is complete

	if (wrap_in && (2 * n_in == L))
		fft512_regs<false, true, SB>(v, s, tw, t, b);
	else
		fft512_regs<false, false, SB>(v, s, tw, t, b);

	const float2* pp = psf + (o % pmod) * pos + cx;
#pragma unroll
	for (int m = 0; m < 32; m++)
		if (valid)
			v[m] = cmul(v[m], pp[(t + 16 * m) * pes]);

	__syncthreads();	// every thread's stage-2 loads are done before s is rewritten
	fft512_regs<true, false, SB>(v, s, tw, t, b);

	if (!valid)
		return;

	float2* outp = out + o * oos + cx;
#pragma unroll
	for (int m = 0; m < 32; m++) {

		const int p = t + 16 * m;
		const int n = wrap_out ? unwrap_pos(p, n_out, L) : p;

		if (n < n_out)
			outp[n * oes] = v[m];
	}
}

// Row pass, inverse --------------------------------------------------------------
//
// Input rows in[p + L*(yz + YZ*c)], p < L. Each block takes B consecutive yz
// rows and coils [c0, c1) (a thread keeps its output pixels in registers
// across the coil loop): inverse FFT per row, keep x < X from
// wrap_pos(x, X, L), scale by ax[x]*ayz[yz] (optional) and either
//   maps != 0: accumulate sum_c conj(maps[x + X*yz + X*YZ*c]) * row
//              into out[x + X*yz + X*YZ*g] (g = blockIdx.y, partial per group)
//   maps == 0: write out[x + X*yz + X*YZ*c] per coil.
// grid (ceil(YZ/B), groups); coils per group cpg.
template <int L, int B, bool BLUE>
__global__ void __launch_bounds__(B * L / 8, (1024 / (B * L / 8)) > 0 ? 1024 / (B * L / 8) : 1) k_rows_inv(const float2* __restrict__ in, const float2* __restrict__ maps,
		const float* __restrict__ ax, const float* __restrict__ ayz,
		int X, long YZ, int C, int cpg, float2* __restrict__ out, const float2* __restrict__ twg,
		const float2* __restrict__ pdot, double* __restrict__ dot_part, const int* done, Dft d)
{
	using LAY = RowLayout<L, B>;
	const int dn = BLUE ? d.n : L;	// logical DFT length (compile-time for the FFT itself)
	constexpr int NT = B * L / 8;
	extern __shared__ float2 smem[];
	__shared__ double red[32];
	float2* s = smem;
	float2* tw = smem + LAY::SMEM;

	if (done && *done)
		return;

	for (int i = threadIdx.x; i < L; i += NT)
		tw[i] = twg[i];

	const long yz = (long)blockIdx.x * B + LAY::seq();
	const bool valid = (yz < YZ);
	const int g = blockIdx.y;
	const int c0 = g * cpg;
	const int c1 = min(C, c0 + cpg);

	// this thread's output pixels: x = unwrap(jt + (L/8) m) where < X
	float2 acc[8];
#pragma unroll
	for (int m = 0; m < 8; m++)
		acc[m] = make_float2(0.f, 0.f);

	double dot = 0.;

	for (int c = c0; c < c1; c++) {

		float2 v[8];
#pragma unroll
		for (int m = 0; m < 8; m++) {

			int p = reg_pos<L, LAY>(m);
			v[m] = (valid && (p < dn)) ? in[p + (long)dn * (yz + YZ * c)] : make_float2(0.f, 0.f);
		}

		dft_regs<L, LAY, true, BLUE>(v, s, tw, d);

		if (valid) {
#pragma unroll
			for (int m = 0; m < 8; m++) {

				int p = reg_pos<L, LAY>(m);
				int x = (p < dn) ? unwrap_pos(p, X, dn) : X;

				if (x >= X)
					continue;

				float2 w = v[m];

				if (ax)
					w = cscale(w, ax[x] * ayz[yz]);

				if (maps) {

					acc[m] = cadd(acc[m], cmulc(w, maps[x + X * yz + X * YZ * c]));

				} else {

					out[x + X * yz + X * YZ * c] = w;

					if (pdot) {	// Re<pdot, out> per coil (pdot == out: ||out||^2)

						float2 pv = ((const void*)pdot == (const void*)out) ? w : pdot[x + X * yz + X * YZ * c];
						dot += (double)pv.x * (double)w.x + (double)pv.y * (double)w.y;
					}
				}
			}
		}
	}

	if (maps) {

		if (valid) {
#pragma unroll
			for (int m = 0; m < 8; m++) {

				int p = reg_pos<L, LAY>(m);
				int x = (p < dn) ? unwrap_pos(p, X, dn) : X;

				if (x >= X)
					continue;

				out[x + X * yz + X * YZ * g] = acc[m];

				if (pdot) {	// Re<p, partial> for the CG step length

					float2 pv = pdot[x + X * yz];
					dot += (double)pv.x * (double)acc[m].x + (double)pv.y * (double)acc[m].y;
				}
			}
		}
	}

	if (pdot) {

		double t = block_sum_d(dot, red);

		if (0 == threadIdx.x)
			dot_part[blockIdx.x + gridDim.x * blockIdx.y] = t;
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
	int G[3];	// grid size per axis (2N, lround(os N) for the chain, or 1)
	long gsz;	// cells per channel
	float hw;	// kernel width on the N-grid (conf.width / 2)
	int periodic;
	// (defaults: the os = 2 gridding, for geometries built field by field)
	int chain = 0;	// os != 2: the chained NUFFT's plain gridding on the G grid
	float os = 2.f;	// its oversampling
	float wg = 6.f;	// its kernel width on the G grid (conf.width)
};

// Taps of one axis of the chained NUFFT (os != 2; nufft_create_chain,
// src/noncart/nufft_chain.c:190-244, gridding by gridH / grid_point_gen,
// src/noncart/grid.c:150-199, 403-465):
//   pos = float(os * k) + float(G/2)   (the centred grid of G cells)
//   taps t = ceil(pos - w/2) .. floor(pos + w/2)  (float64 bounds)
//   weight = intlookup(|t - pos| / w)
//   cell: centred t -> DFT order (t + G/2) mod G (G even)
// Non-periodic: taps clipped to [0, G-1]; periodic: t mod G.
__device__ __forceinline__ void chain_taps(float k, int G, float os, float w, int periodic, const float* kb,
		AxisTaps& t)
{
	t.n = 0;

	if (1 == G) {

		t.cell[0] = 0;
		t.w[0] = kb_lookup(kb, 0.f);
		t.n = 1;
		return;
	}

	const float pos = __fadd_rn(__fmul_rn(os, k), (float)(G / 2));
	int sti = (int)ceil((double)pos - 0.5 * (double)w);
	int eni = (int)floor((double)pos + 0.5 * (double)w);

	if (!periodic) {

		sti = max(sti, 0);
		eni = min(eni, G - 1);
	}

	for (int c = sti; (c <= eni) && (t.n < MAX_AXIS_TAPS); c++) {

		const float frac = fabsf(__fsub_rn((float)c, pos));
		const int cm = periodic ? (((c % G) + G) % G) : c;
		int j = cm + G / 2;

		if (j >= G)
			j -= G;

		t.cell[t.n] = j;
		t.w[t.n] = kb_lookup(kb, __fdiv_rn(frac, w));
		t.n++;
	}
}

// the taps of axis a for either gridding
__device__ __forceinline__ void geom_taps(const GridGeom& g, int a, float k, const float* kb, AxisTaps& t)
{
	if (g.chain)
		chain_taps(k, g.G[a], g.os, g.wg, g.periodic, kb, t);
	else
		axis_taps(k, g.N[a], g.hw, g.periodic, kb, t);
}

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
	geom_taps(g, 0, k.x, kb, tx);
	geom_taps(g, 1, k.y, kb, ty);
	geom_taps(g, 2, k.z, kb, tz);

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
	geom_taps(g, 0, k.x, kb, tx);
	geom_taps(g, 1, k.y, kb, ty);
	geom_taps(g, 2, k.z, kb, tz);

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

// Deterministic gridding --------------------------------------------------------
//
// The adjoint interpolation as a sparse matrix in CSR form over grid cells:
// row = cell, entries (sample, weight) in increasing sample order. It is
// built once per trajectory (k_csr_keys + a stable radix sort by
// cell * M + sample + k_csr_fill), after which gridding is a gather per
// cell in that fixed order: no atomics, bit-identical results run to run,
// and every cell is written (no clearing pass). The weights are the same
// float32 products as in k_grid_atomic.

enum { CSR_TAPS_AXIS = 8 };	// per axis: two sub-grids x up to 4 taps (width <= 6)

// one key (cell * M + m, or ~0 for an unused slot) and weight per (sample, tap slot)
__global__ void k_csr_keys(const float4* __restrict__ traj, long M, GridGeom g, const float* __restrict__ kbg,
		unsigned long long* __restrict__ keys, float* __restrict__ vals, int slots_z)
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
	geom_taps(g, 0, k.x, kb, tx);
	geom_taps(g, 1, k.y, kb, ty);
	geom_taps(g, 2, k.z, kb, tz);

	const int slots = CSR_TAPS_AXIS * CSR_TAPS_AXIS * slots_z;
	unsigned long long* kp = keys + m * slots;
	float* vp = vals + m * slots;
	int t = 0;

	for (int a = 0; a < tz.n; a++) {

		float dz = tz.w[a];
		long oz = (long)tz.cell[a] * g.G[1];

		for (int bb = 0; bb < ty.n; bb++) {

			float dzy = __fmul_rn(dz, ty.w[bb]);
			long oy = (oz + ty.cell[bb]) * g.G[0];

			for (int cc = 0; cc < tx.n; cc++) {

				if (t < slots) {

					kp[t] = (unsigned long long)(oy + tx.cell[cc]) * (unsigned long long)M + (unsigned long long)m;
					vp[t] = __fmul_rn(dzy, tx.w[cc]);
					t++;
				}
			}
		}
	}

	for (; t < slots; t++) {

		kp[t] = ~0ull;
		vp[t] = 0.f;
	}
}

// sorted keys -> column (sample) indices and per-cell counts; unused slots
// (key ~0) sort to the end and are not counted
__global__ void k_csr_fill_valid(const unsigned long long* __restrict__ keys, long nnz, long M, long gsz,
		int* __restrict__ col, int* __restrict__ counts)
{
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += (long)gridDim.x * blockDim.x) {

		unsigned long long key = keys[i];

		if (~0ull == key) {

			col[i] = 0;
			continue;
		}

		long cell = (long)(key / (unsigned long long)M);
		col[i] = (int)(key % (unsigned long long)M);

		if (cell < gsz)
			atomicAdd(&counts[cell], 1);	// integer counts: order-independent
	}
}

// grid[cell + gsz*c] = sum over the cell's row of w * ksp[m + M*c]: one warp
// per cell, lane l sums entries l, l+32, ... in order, then a fixed shuffle
// tree combines the lanes, so the summation order is the same every run (and
// long rows at the k-space centre are spread over 32 lanes).
__global__ void k_grid_csr(const long* __restrict__ row_ptr, const int* __restrict__ col, const float* __restrict__ val,
		long gsz, long M, int C, int cpc, const float2* __restrict__ ksp, float2* __restrict__ grid)
{
	const int lane = threadIdx.x % 32;
	long cell = ((long)blockIdx.x * blockDim.x + threadIdx.x) / 32;

	if (cell >= gsz)
		return;

	const long r0 = row_ptr[cell];
	const long r1 = row_ptr[cell + 1];
	const int c0 = blockIdx.y * cpc;
	const int c1 = min(C, c0 + cpc);

	for (int cb = c0; cb < c1; cb += 4) {

		float2 acc[4];
#pragma unroll
		for (int q = 0; q < 4; q++)
			acc[q] = make_float2(0.f, 0.f);

		for (long i = r0 + lane; i < r1; i += 32) {

			float w = val[i];
			long m = col[i];
#pragma unroll
			for (int q = 0; q < 4; q++) {

				if (cb + q < c1) {

					float2 y = ksp[m + M * (cb + q)];
					acc[q].x = fmaf(y.x, w, acc[q].x);
					acc[q].y = fmaf(y.y, w, acc[q].y);
				}
			}
		}

#pragma unroll
		for (int q = 0; q < 4; q++) {

			for (int o = 16; o > 0; o >>= 1) {

				acc[q].x += __shfl_xor_sync(0xffffffffu, acc[q].x, o);
				acc[q].y += __shfl_xor_sync(0xffffffffu, acc[q].y, o);
			}

			if ((0 == lane) && (cb + q < c1))
				grid[cell + gsz * (cb + q)] = acc[q];
		}
	}
}

} // namespace bn
