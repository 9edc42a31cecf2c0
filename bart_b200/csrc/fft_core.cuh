// Shared-memory Stockham FFT core for sm_100a.
//
// A thread block transforms B sequences of length L (power of two, 16..4096).
// Each sequence is served by T = L/8 threads (index jt). Between stages the
// data lives in shared memory in one of two layouts (ColLayout for column
// passes, RowLayout for row passes; see below), chosen so that both the
// global accesses and the shared-memory stages stay conflict-free. Stages are
// radix 8 with a final radix 4 or 2 (Stockham autosort, so the result is in
// natural order without a bit-reversal pass).
//
// Register ownership: before the first stage and after the last stage a
// thread holds the eight elements at positions jt + T*m (m = 0..7) in
// v[m]. The first stage reads exactly these positions and the last stage
// writes them, so the caller loads stage-1 input straight from global memory
// and consumes the last-stage output in registers (e.g. the Toeplitz PSF
// product between a forward and an inverse transform needs no shared-memory
// pass at all).
//
// Forward = exp(-2 pi i jk / L), inverse = exp(+2 pi i jk / L), unnormalised,
// as FFTW's / the reference's FFT (src/num/fft_plan.c:227). Twiddles come
// from a table tw[m] = exp(-2 pi i m / L) computed on the host in float64.
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

// dft8 of (v0, v1, 0, 0, 0, 0, v6, v7): the first stage of a transform whose
// input is zero-padded to twice its length with the centred placement (the
// nonzero half at positions < L/4 and >= 3L/4, i.e. registers 0, 1, 6, 7).
// The same operations as dft8 minus those on the known zeros, so the same
// results (up to the sign of exact zeros).
template <bool INV>
__device__ __forceinline__ void dft8_half(float2* v)
{
	// dft4 of (a, 0, 0, b): (a + b, a + rot(-b), a - b, a - rot(-b))
	const float2 e0 = cadd(v[0], v[6]), e2 = csub(v[0], v[6]);
	const float2 eb = rot90<INV>(make_float2(-v[6].x, -v[6].y));
	const float2 e1 = cadd(v[0], eb), e3 = csub(v[0], eb);
	const float2 o0 = cadd(v[1], v[7]), o2 = csub(v[1], v[7]);
	const float2 ob = rot90<INV>(make_float2(-v[7].x, -v[7].y));
	const float2 o1 = cadd(v[1], ob), o3 = csub(v[1], ob);
	const float c = 0.70710678118654752440f;
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

// twiddle v[i] *= w^(i*k), w = exp(-+2 pi i / (Ns*R)): w^k from the table
// tw[m] = exp(-2 pi i m / L), its powers by complex multiplication (one
// shared-memory load per stage instead of R - 1; the products add a few
// float32 roundings, well below the transforms' own error)
template <int L, int Ns, int R, bool INV>
__device__ __forceinline__ void twiddle(float2* v, int k, const float2* tw)
{
	if constexpr (Ns > 1) {

		float2 w1 = tw[k * (L / (Ns * R))];

		if (INV)
			w1.y = -w1.y;

		float2 w = w1;
#pragma unroll
		for (int i = 1; i < R; i++) {

			v[i] = cmul(v[i], w);

			if (i + 1 < R)
				w = cmul(w, w1);
		}
	}
}

// Shared-memory layouts of B sequences of length L (element indices).
//
// ColLayout: sequences interleaved, element p of sequence b at p*SB + b
// (SB = B|1 odd, so a half-warp's 8-byte accesses hit distinct banks);
// thread t serves sequence t % B with index t / B. A warp covers the same
// element of consecutive sequences: coalesced for columns of an x-fastest
// array.
template <int L, int B>
struct ColLayout {

	static constexpr int SB = B | 1;
	static constexpr int SMEM = L * SB;

	__device__ static __forceinline__ int idx(int p, int b) { return p * SB + b; }
	__device__ static __forceinline__ int seq() { return threadIdx.x % B; }
	__device__ static __forceinline__ int jt() { return threadIdx.x / B; }
};

// RowLayout: each sequence contiguous with one pad element after every 8
// (p + p/8 breaks the stride-8 bank pattern of the first stage's stores);
// thread t serves sequence t / (L/8) with index t % (L/8). A warp covers
// consecutive elements of one sequence: coalesced for contiguous rows.
template <int L, int B>
struct RowLayout {

	static constexpr int SL = L + L / 8;
	static constexpr int SMEM = B * SL;

	__device__ static __forceinline__ int idx(int p, int b) { return b * SL + p + (p >> 3); }
	__device__ static __forceinline__ int seq() { return threadIdx.x / (L / 8); }
	__device__ static __forceinline__ int jt() { return threadIdx.x % (L / 8); }
};

// Stage with Ns = product of earlier radices, Ns > 1: smem -> smem (middle
// stages) or smem -> registers (the last stage).
template <int L, typename LAY, int Ns, bool INV>
__device__ __forceinline__ void fft_tail(float2 (&v)[8], float2* s, int b, int jt, const float2* tw)
{
	constexpr int REM = L / Ns;
	constexpr int R = (REM >= 8) ? 8 : REM;
	constexpr int NB = L / R;
	constexpr int T = L / 8;
	constexpr int PER = NB / T;
	constexpr bool LAST = (Ns * R == L);

	float2 u[PER][R];

#pragma unroll
	for (int q = 0; q < PER; q++) {
#pragma unroll
		for (int i = 0; i < R; i++)
			u[q][i] = s[LAY::idx(jt + q * T + i * NB, b)];
	}

	if constexpr (!LAST)
		__syncthreads();

#pragma unroll
	for (int q = 0; q < PER; q++) {

		int j = jt + q * T;
		int k = j % Ns;
		twiddle<L, Ns, R, INV>(u[q], k, tw);
		butterfly<R, INV>(u[q]);

		if constexpr (LAST) {
			// outputs at j + NB*i = jt + T*(q + PER*i)
#pragma unroll
			for (int i = 0; i < R; i++)
				v[q + PER * i] = u[q][i];

		} else {

			int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
			for (int i = 0; i < R; i++)
				s[LAY::idx(idxD + i * Ns, b)] = u[q][i];
		}
	}

	if constexpr (!LAST) {

		__syncthreads();
		fft_tail<L, LAY, Ns * R, INV>(v, s, b, jt, tw);
	}
}

// Full transform of the register set v (positions jt + (L/8)*m in, same
// out). Begins with a barrier, so the caller may have been reading s just
// before; the caller must barrier before writing s after it returns.
// half_in: registers 2..5 are known zeros (input of length L/2, centred).
template <int L, typename LAY, bool INV>
__device__ __forceinline__ void fft_regs(float2 (&v)[8], float2* s, const float2* tw, bool half_in = false)
{
	static_assert(L >= 16 && L <= 4096 && (L & (L - 1)) == 0, "power-of-two length 16..4096");
	const int b = LAY::seq();
	const int jt = LAY::jt();

	// stage 1 (Ns = 1, radix 8, no twiddles): registers -> smem at 8*jt + i
	if (half_in)
		dft8_half<INV>(v);
	else
		butterfly<8, INV>(v);
	__syncthreads();
#pragma unroll
	for (int i = 0; i < 8; i++)
		s[LAY::idx(8 * jt + i, b)] = v[i];
	__syncthreads();

	fft_tail<L, LAY, 8, INV>(v, s, b, jt, tw);
}

// Double-buffered form for transforms of three stages (L = 128, 256, 512):
// stage 1 writes s, stage 2 reads s and writes s2, stage 3 reads s2. Each
// stage writes a buffer that no thread reads any more (the other one was
// read in the stage before, which every thread finished before the last
// barrier), so one barrier per exchange suffices and the transform needs no
// barrier on entry: two transforms in a row (forward, then inverse) are
// safe, since the second one's stage 1 writes s, last read in the first
// one's stage 2. Same arithmetic as fft_regs, so the same results.
template <int L, typename LAY, int Ns, bool INV>
__device__ __forceinline__ void fft_tail_db(float2 (&v)[8], const float2* sr, float2* sw, int b, int jt,
		const float2* tw)
{
	constexpr int REM = L / Ns;
	constexpr int R = (REM >= 8) ? 8 : REM;
	constexpr int NB = L / R;
	constexpr int T = L / 8;
	constexpr int PER = NB / T;
	constexpr bool LAST = (Ns * R == L);

	float2 u[PER][R];

#pragma unroll
	for (int q = 0; q < PER; q++) {
#pragma unroll
		for (int i = 0; i < R; i++)
			u[q][i] = sr[LAY::idx(jt + q * T + i * NB, b)];
	}

#pragma unroll
	for (int q = 0; q < PER; q++) {

		int j = jt + q * T;
		int k = j % Ns;
		twiddle<L, Ns, R, INV>(u[q], k, tw);
		butterfly<R, INV>(u[q]);

		if constexpr (LAST) {
#pragma unroll
			for (int i = 0; i < R; i++)
				v[q + PER * i] = u[q][i];

		} else {

			int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
			for (int i = 0; i < R; i++)
				sw[LAY::idx(idxD + i * Ns, b)] = u[q][i];
		}
	}

	if constexpr (!LAST) {

		__syncthreads();
		fft_tail_db<L, LAY, Ns * R, INV>(v, sw, const_cast<float2*>(sr), b, jt, tw);
	}
}

template <int L, typename LAY, bool INV>
__device__ __forceinline__ void fft_regs_db(float2 (&v)[8], float2* s, float2* s2, const float2* tw,
		bool half_in = false)
{
	static_assert((L >= 128) && (L <= 512), "three-stage lengths only");
	const int b = LAY::seq();
	const int jt = LAY::jt();

	if (half_in)
		dft8_half<INV>(v);
	else
		butterfly<8, INV>(v);
#pragma unroll
	for (int i = 0; i < 8; i++)
		s[LAY::idx(8 * jt + i, b)] = v[i];
	__syncthreads();

	fft_tail_db<L, LAY, 8, INV>(v, s, s2, b, jt, tw);
}

// stage-1 position of register m for this thread
template <int L, typename LAY>
__device__ __forceinline__ int reg_pos(int m) { return LAY::jt() + (L / 8) * m; }

} // namespace bn
