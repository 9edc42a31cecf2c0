// Shared-memory Stockham FFT core for sm_100a.
//
// A thread block transforms B sequences of length L (power of two, 16..2048)
// held in shared memory as s[p * SB + b] (element p of sequence b; SB = B|1 so
// that the element stride is odd and 8-byte accesses of a half-warp hit
// distinct banks). Each sequence is served by L/8 threads; one radix-8 (or a
// final radix-4/2) butterfly per thread per stage, autosorting (Stockham), so
// the result lands in natural order without a bit-reversal pass.
//
// Forward = exp(-2 pi i jk / L), inverse = exp(+2 pi i jk / L), both
// unnormalised, as FFTW's / the reference's FFT (src/num/fft_plan.c:227).
// Twiddles come from a table tw[m] = exp(-2 pi i m / L) computed on the host
// in float64, so the transform is accurate to a few float32 ulps.
#pragma once

#include <cuda_runtime.h>

namespace bn {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
	return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b)
{
	return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 rot90(float2 a)
{
	return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <bool INV>
__device__ __forceinline__ void dft2(float2* v)
{
	float2 a = v[0];
	v[0] = cadd(a, v[1]);
	v[1] = csub(a, v[1]);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& v0, float2& v1, float2& v2, float2& v3)
{
	float2 a0 = cadd(v0, v2), a1 = csub(v0, v2);
	float2 a2 = cadd(v1, v3), a3 = rot90<INV>(csub(v1, v3));
	v0 = cadd(a0, a2);
	v2 = csub(a0, a2);
	v1 = cadd(a1, a3);
	v3 = csub(a1, a3);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2* v) { dft4<INV>(v[0], v[1], v[2], v[3]); }

template <bool INV>
__device__ __forceinline__ void dft8(float2* v)
{
	// decimation in time: two length-4 DFTs, then W8^k twiddles and a radix-2 combine
	float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
	float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
	dft4<INV>(e0, e1, e2, e3);
	dft4<INV>(o0, o1, o2, o3);
	const float c = 0.70710678118654752440f;
	// W8^1 = (c, -+c), W8^2 = -+i, W8^3 = (-c, -+c)
	float2 t1 = INV ? make_float2(c * (o1.x - o1.y), c * (o1.x + o1.y))
			: make_float2(c * (o1.x + o1.y), c * (o1.y - o1.x));
	float2 t2 = rot90<INV>(o2);
	float2 t3 = INV ? make_float2(-c * (o3.x + o3.y), c * (o3.x - o3.y))
			: make_float2(c * (o3.y - o3.x), -c * (o3.x + o3.y));
	v[0] = cadd(e0, o0);
	v[4] = csub(e0, o0);
	v[1] = cadd(e1, t1);
	v[5] = csub(e1, t1);
	v[2] = cadd(e2, t2);
	v[6] = csub(e2, t2);
	v[3] = cadd(e3, t3);
	v[7] = csub(e3, t3);
}

template <int R, bool INV>
__device__ __forceinline__ void butterfly(float2* v)
{
	if constexpr (R == 8)
		dft8<INV>(v);
	else if constexpr (R == 4)
		dft4<INV>(v);
	else
		dft2<INV>(v);
}

// One Stockham stage per recursion level; Ns = product of the radices done.
template <int L, int Ns, bool INV>
__device__ __forceinline__ void fft_stages(float2* s, int SB, int b, int jt, const float2* tw)
{
	if constexpr (Ns < L) {

		constexpr int REM = L / Ns;
		constexpr int R = (REM >= 8) ? 8 : REM;
		constexpr int NB = L / R;	// butterflies per sequence
		constexpr int T = L / 8;	// threads per sequence
		constexpr int PER = NB / T;	// butterflies per thread this stage

		float2 v[PER][R];

#pragma unroll
		for (int q = 0; q < PER; q++) {

			int j = jt + q * T;
#pragma unroll
			for (int i = 0; i < R; i++)
				v[q][i] = s[(j + i * NB) * SB + b];
		}

		__syncthreads();

#pragma unroll
		for (int q = 0; q < PER; q++) {

			int j = jt + q * T;
			int k = j & (Ns - 1);

			if constexpr (Ns > 1) {
#pragma unroll
				for (int i = 1; i < R; i++) {

					float2 w = tw[i * k * (L / (Ns * R))];
					if (INV)
						w.y = -w.y;
					v[q][i] = cmul(v[q][i], w);
				}
			}

			butterfly<R, INV>(v[q]);

			int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
			for (int i = 0; i < R; i++)
				s[(idxD + i * Ns) * SB + b] = v[q][i];
		}

		__syncthreads();

		fft_stages<L, Ns * R, INV>(s, SB, b, jt, tw);
	}
}

// Transform all B sequences in s. Must be called by exactly B * L / 8 threads
// (the whole block), thread t serving sequence t % B.
template <int L, bool INV>
__device__ __forceinline__ void fft_block(float2* s, int SB, int B, const float2* tw)
{
	static_assert(L >= 16 && (L & (L - 1)) == 0, "power-of-two length >= 16");
	int b = threadIdx.x % B;
	int jt = threadIdx.x / B;
	fft_stages<L, 1, INV>(s, SB, b, jt, tw);
}

} // namespace bn
