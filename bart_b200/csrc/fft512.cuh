// 512-point transforms in two stages (16 x 32) for the Toeplitz column pass.
//
// X[k1 + 16 k2] = sum_n2 W32^(n2 k2) W512^(n2 k1) sum_n1 W16^(n1 k1) x[32 n1 + n2]
// (the four-step factorisation, n = 32 n1 + n2). Sixteen threads serve one
// sequence; thread t holds the 32 elements at positions t + 16 m (m =
// 0..31) in v[m] before and after a transform:
//   stage 1: for n2 = t and t + 16 (the elements v[2 n1 + h], h = 0, 1) a
//            16-point DFT over n1, times W512^(n2 k1), to shared memory at
//            (k1, n2);
//   stage 2: thread t reads row k1 = t, a 32-point DFT over n2 gives
//            X[t + 16 k2] = v[k2].
// So a transform has one shared-memory exchange and one barrier, and
// forward and inverse transforms chain in registers (the PSF product sits
// between them). The 16- and 32-point DFTs are radix-4 x 4 and 8 x 4 with
// twiddles from the exact constants below; W512 powers come from the
// float64-built table tw (tw[m] = exp(-2 pi i m / 512)): two loads per
// 16 twiddles, the rest by complex products.
#pragma once

#include <cuda_runtime.h>

#include "fft_core.cuh"

namespace bn {

// exp(-2 pi i k / 32) for k = 0..31 (float32 of the float64 values; the
// axis points exact)
__device__ __forceinline__ float2 w32_const(int k)
{
	constexpr float C[8] = { 1.0f, 9.807852507e-1f, 9.238795042e-1f, 8.314695954e-1f,
				 7.071067691e-1f, 5.555702448e-1f, 3.826834261e-1f, 1.950903237e-1f };
	constexpr float S[8] = { 0.0f, 1.950903237e-1f, 3.826834261e-1f, 5.555702448e-1f,
				 7.071067691e-1f, 8.314695954e-1f, 9.238795042e-1f, 9.807852507e-1f };
	k &= 31;
	const int q = k >> 3, r = k & 7;	// quadrant, offset

	// exp(-i (2 pi / 32) (8 q + r)) = (-i)^q (C_r - i S_r)
	const float c = C[r], s = S[r];

	switch (q) {
	case 0: return make_float2(c, -s);
	case 1: return make_float2(-s, -c);
	case 2: return make_float2(-c, s);
	default: return make_float2(s, c);
	}
}

// a * W32^k (forward) or a * conj(W32^k) (inverse); k known at compile time
// after unrolling; quarter turns exact
template <bool INV>
__device__ __forceinline__ float2 mul_w32(float2 a, int k)
{
	k &= 31;

	if (0 == k)
		return a;

	if (8 == k)
		return rot90<INV>(a);

	if (16 == k)
		return make_float2(-a.x, -a.y);

	if (24 == k)
		return rot90<!INV>(a);

	float2 w = w32_const(k);

	if (INV)
		w.y = -w.y;

	return cmul(a, w);
}

// 16-point DFT of u (natural order in and out). ZERO: u[4..11] are known
// zeros (the first stage of a transform of a 2x zero-padded centred input);
// the same operations minus those on the zeros.
template <bool INV, bool ZERO>
__device__ __forceinline__ void dft16(float2 (&u)[16])
{
	float2 y[16];	// y[b + 4 c]: stage A output of column b, frequency c
#pragma unroll
	for (int b = 0; b < 4; b++) {

		float2 a0 = u[b], a1 = u[b + 4], a2 = u[b + 8], a3 = u[b + 12];

		if (ZERO) {	// a1 = a2 = 0: dft4 of (a0, 0, 0, a3)

			const float2 r3 = rot90<INV>(a3);	// a3 * W4^1
			y[b + 0] = cadd(a0, a3);
			y[b + 4] = csub(a0, r3);		// a0 + a3 W4^3 = a0 - a3 W4^1
			y[b + 8] = csub(a0, a3);
			y[b + 12] = cadd(a0, r3);

		} else {

			dft4<INV>(a0, a1, a2, a3);
			y[b + 0] = a0;
			y[b + 4] = a1;
			y[b + 8] = a2;
			y[b + 12] = a3;
		}
	}

#pragma unroll
	for (int b = 1; b < 4; b++)
#pragma unroll
		for (int c = 1; c < 4; c++)
			y[b + 4 * c] = mul_w32<INV>(y[b + 4 * c], 2 * b * c);	// W16^(b c)

#pragma unroll
	for (int c = 0; c < 4; c++) {

		float2 a0 = y[4 * c + 0], a1 = y[4 * c + 1], a2 = y[4 * c + 2], a3 = y[4 * c + 3];
		dft4<INV>(a0, a1, a2, a3);
		u[c + 0] = a0;		// X[c + 4 d] for d = 0..3
		u[c + 4] = a1;
		u[c + 8] = a2;
		u[c + 12] = a3;
	}
}

// 32-point DFT of u (natural order in and out): radix 8 x 4
template <bool INV>
__device__ __forceinline__ void dft32(float2 (&u)[32])
{
	float2 y[32];	// y[b + 4 c]: stage A (8-point DFT over a of u[4 a + b]) output c of column b
#pragma unroll
	for (int b = 0; b < 4; b++) {

		float2 t[8];
#pragma unroll
		for (int a = 0; a < 8; a++)
			t[a] = u[4 * a + b];

		dft8<INV>(t);
#pragma unroll
		for (int c = 0; c < 8; c++)
			y[b + 4 * c] = (b > 0 && c > 0) ? mul_w32<INV>(t[c], b * c) : t[c];
	}

#pragma unroll
	for (int c = 0; c < 8; c++) {

		float2 a0 = y[4 * c + 0], a1 = y[4 * c + 1], a2 = y[4 * c + 2], a3 = y[4 * c + 3];
		dft4<INV>(a0, a1, a2, a3);
		u[c + 0] = a0;		// X[c + 8 d] for d = 0..3
		u[c + 8] = a1;
		u[c + 16] = a2;
		u[c + 24] = a3;
	}
}

// W512^(n2 k1) for k1 = 0..15 into w[k1] (inverse: conjugated): two table
// loads (w^1, w^4) and products of short chains
template <bool INV>
__device__ __forceinline__ void w512_powers(const float2* tw, int n2, float2 (&w)[16])
{
	float2 w1 = tw[n2 & 511];
	float2 w4 = tw[(4 * n2) & 511];

	if (INV) {

		w1.y = -w1.y;
		w4.y = -w4.y;
	}

	const float2 w2 = cmul(w1, w1), w3 = cmul(w2, w1);
	const float2 w8 = cmul(w4, w4), w12 = cmul(w8, w4);
	const float2 base[4] = { make_float2(1.f, 0.f), w4, w8, w12 };
	const float2 off[4] = { make_float2(1.f, 0.f), w1, w2, w3 };
#pragma unroll
	for (int q = 0; q < 4; q++)
#pragma unroll
		for (int r = 0; r < 4; r++)
			w[4 * q + r] = (0 == q) ? off[r] : ((0 == r) ? base[q] : cmul(base[q], off[r]));
}

// One 512-point transform of the register set v (positions t + 16 m). The
// exchange buffer s holds the block's sequences as s[p * SB + b] (p =
// k1 * 32 + n2). Barriers: one between the stage-1 stores and the stage-2
// loads; the caller puts one before the next stores into s. ZERO: positions
// 128..383 are known zeros (2x zero-padded centred input).
template <bool INV, bool ZERO, int SB>
__device__ __forceinline__ void fft512_regs(float2 (&v)[32], float2* s, const float2* tw, int t, int b)
{
#pragma unroll
	for (int h = 0; h < 2; h++) {

		float2 u[16];
#pragma unroll
		for (int n1 = 0; n1 < 16; n1++)
			u[n1] = v[2 * n1 + h];

		dft16<INV, ZERO>(u);
		const int n2 = t + 16 * h;
		float2 w[16];
		w512_powers<INV>(tw, n2, w);
#pragma unroll
		for (int k1 = 0; k1 < 16; k1++)
			s[(k1 * 32 + n2) * SB + b] = (0 == k1) ? u[0] : cmul(u[k1], w[k1]);
	}

	__syncthreads();

	float2 r[32];
#pragma unroll
	for (int n2 = 0; n2 < 32; n2++)
		r[n2] = s[(t * 32 + n2) * SB + b];

	dft32<INV>(r);
#pragma unroll
	for (int k2 = 0; k2 < 32; k2++)
		v[k2] = r[k2];
}

} // namespace bn
