// Learned preconditioner for flexible CG: a 6-layer 3x3 convolutional
// network on one complex image (real and imaginary parts as 2 channels),
// 2 -> 32 -> 32 -> 32 -> 32 -> 32 -> 2 channels, ReLU after layers 1-5,
// zero padding. Weights are bfloat16, accumulation float32.
//
// Activations are bfloat16 in NHWC order, 32 channels per pixel
// (act[((img * Y + y) * X + x) * 32 + c]), pixel (x, y) of a BART image
// [X, Y] (x fastest). Layers 2-5 run on the tensor cores (mma.sync
// m16n8k16 bf16 -> f32): a block computes a 32 x 8 pixel tile of all 32
// output channels as a GEMM of the tile's im2col rows (K = 9 taps x 32
// channels) with the weight matrix, both staged in shared memory. Layers 1
// and 6 (2 input / 2 output channels) are thin and run on the FP32 pipes.
//
// Training uses the same kernels plus the backward passes: the data
// gradient of a 32 -> 32 layer is the forward kernel with the weights
// transposed and the taps flipped, masked by the ReLU of the layer below;
// weight gradients are FP32 sums over pixels, per block, then reduced in a
// fixed order (bit-reproducible).
//
// Parameter vector (float32), per layer l = 1..6: W_l[cout][tap][cin]
// (tap = 3 ky + kx), then b_l[cout].
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "nufft_kernels.cuh"

namespace bn {

typedef __nv_bfloat16 bf16;
typedef __nv_bfloat162 bf162;

enum { NET_C = 32, NET_TILE_X = 32, NET_TILE_Y = 8, NET_THREADS = 256 };

constexpr int NET_SA_STRIDE = 40;	// bf16 per pixel in the halo tile (32 + 8 pad: conflict-free fragments)
constexpr int NET_SW_STRIDE = 296;	// bf16 per output channel in the weight tile (288 + 8 pad)
constexpr int NET_HALO_X = NET_TILE_X + 2, NET_HALO_Y = NET_TILE_Y + 2;
constexpr size_t NET_CONV_SMEM = sizeof(bf16) * (NET_HALO_X * NET_HALO_Y * NET_SA_STRIDE + NET_C * NET_SW_STRIDE);

struct NetLayout {

	// parameter offsets of W_l and b_l, l = 0..5
	__host__ __device__ static constexpr int cin(int l) { return (0 == l) ? 2 : NET_C; }
	__host__ __device__ static constexpr int cout(int l) { return (5 == l) ? 2 : NET_C; }
	__host__ __device__ static constexpr int wsize(int l) { return cout(l) * 9 * cin(l); }
	__host__ __device__ static constexpr int size(int l) { return wsize(l) + cout(l); }
	__host__ __device__ static constexpr int woff(int l) { return (0 == l) ? 0 : woff(l - 1) + size(l - 1); }
	__host__ __device__ static constexpr int boff(int l) { return woff(l) + wsize(l); }
	__host__ __device__ static constexpr int total() { return woff(5) + size(5); }
};

static_assert(NetLayout::total() == 38178, "parameter count");

__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
		uint32_t b0, uint32_t b1)
{
	asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
		"{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
		: "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
		: "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t lds32(const bf16* p) { return *(const uint32_t*)p; }

// 32 -> 32 channel 3x3 convolution on the tensor cores.
//   MODE 0 (forward):  out = bf16(relu(conv(in, w) + bias))
//   MODE 1 (backward): out = bf16(conv(in, w) * (mask > 0)), with in = the
//                      gradient of the layer above and w its transposed,
//                      tap-flipped weights.
// w: bf16 [32 cout][9 tap][32 cin]. grid (ceil(X/32), ceil(Y/8), nimg).
template <int MODE>
__global__ void __launch_bounds__(NET_THREADS) k_conv32(const bf16* __restrict__ in, const bf16* __restrict__ w,
		const float* __restrict__ bias, const bf16* __restrict__ mask, bf16* __restrict__ out, int X, int Y,
		const int* done, const int* skip = nullptr)
{
	extern __shared__ __align__(16) unsigned char net_smem[];
	bf16* sA = (bf16*)net_smem;
	bf16* sW = sA + NET_HALO_X * NET_HALO_Y * NET_SA_STRIDE;

	if ((done && *done) || (skip && *skip))
		return;

	const int x0 = blockIdx.x * NET_TILE_X;
	const int y0 = blockIdx.y * NET_TILE_Y;
	const long ibase = (long)blockIdx.z * X * Y;

	// weights: 32 rows of 288 bf16 = 36 x 16 B
	for (int i = threadIdx.x; i < NET_C * 36; i += NET_THREADS) {

		int co = i / 36;
		int j = i % 36;
		*(uint4*)(sW + co * NET_SW_STRIDE + j * 8) = ((const uint4*)(w + co * 288))[j];
	}

	// halo tile: 10 x 34 pixels, 64 B each (4 x 16 B), zero outside the image
	for (int i = threadIdx.x; i < NET_HALO_X * NET_HALO_Y * 4; i += NET_THREADS) {

		int q = i & 3;
		int pix = i >> 2;
		int gy = y0 + pix / NET_HALO_X - 1;
		int gx = x0 + pix % NET_HALO_X - 1;
		uint4 v = make_uint4(0u, 0u, 0u, 0u);

		if ((gy >= 0) && (gy < Y) && (gx >= 0) && (gx < X))
			v = ((const uint4*)(in + (ibase + (long)gy * X + gx) * NET_C))[q];

		*(uint4*)(sA + pix * NET_SA_STRIDE + q * 8) = v;
	}

	__syncthreads();

	const int warp = threadIdx.x >> 5;	// tile row
	const int lane = threadIdx.x & 31;
	const int g = lane >> 2;
	const int t = lane & 3;

	float acc[2][4][4];
#pragma unroll
	for (int mt = 0; mt < 2; mt++)
#pragma unroll
		for (int nt = 0; nt < 4; nt++)
#pragma unroll
			for (int e = 0; e < 4; e++)
				acc[mt][nt][e] = 0.f;

#pragma unroll 1
	for (int tap = 0; tap < 9; tap++) {

		const int ky = tap / 3;
		const int kx = tap % 3;
#pragma unroll
		for (int h = 0; h < 2; h++) {	// input channels 16 h .. 16 h + 15

			uint32_t b[4][2];
#pragma unroll
			for (int nt = 0; nt < 4; nt++) {

				const bf16* wp = sW + (nt * 8 + g) * NET_SW_STRIDE + tap * NET_C + h * 16 + 2 * t;
				b[nt][0] = lds32(wp);
				b[nt][1] = lds32(wp + 8);
			}
#pragma unroll
			for (int mt = 0; mt < 2; mt++) {

				const bf16* ap = sA + ((warp + ky) * NET_HALO_X + mt * 16 + g + kx) * NET_SA_STRIDE + h * 16 + 2 * t;
				uint32_t a0 = lds32(ap);
				uint32_t a1 = lds32(ap + 8 * NET_SA_STRIDE);
				uint32_t a2 = lds32(ap + 8);
				uint32_t a3 = lds32(ap + 8 * NET_SA_STRIDE + 8);
#pragma unroll
				for (int nt = 0; nt < 4; nt++)
					mma_bf16(acc[mt][nt], a0, a1, a2, a3, b[nt][0], b[nt][1]);
			}
		}
	}

	const int gy = y0 + warp;

	if (gy >= Y)
		return;

#pragma unroll
	for (int mt = 0; mt < 2; mt++) {
#pragma unroll
		for (int hh = 0; hh < 2; hh++) {

			const int gx = x0 + mt * 16 + g + 8 * hh;

			if (gx >= X)
				continue;

			const long o = (ibase + (long)gy * X + gx) * NET_C;
#pragma unroll
			for (int nt = 0; nt < 4; nt++) {

				const int co = nt * 8 + 2 * t;
				float v0 = acc[mt][nt][2 * hh];
				float v1 = acc[mt][nt][2 * hh + 1];

				if (0 == MODE) {

					v0 = fmaxf(v0 + bias[co], 0.f);
					v1 = fmaxf(v1 + bias[co + 1], 0.f);

				} else {

					bf162 m = *(const bf162*)(mask + o + co);
					v0 = (__bfloat162float(m.x) > 0.f) ? v0 : 0.f;
					v1 = (__bfloat162float(m.y) > 0.f) ? v1 : 0.f;
				}

				*(bf162*)(out + o + co) = __floats2bfloat162_rn(v0, v1);
			}
		}
	}
}

// Layer 1 (2 -> 32), one thread per pixel: act = bf16(relu(conv(s * in) + b)),
// in complex [nimg][Y][X], s = *scale, or 1 / sqrt(sum of norm_part) (the
// input's norm from the partials of the pass that wrote it), or 1. w: float
// [32][9][2] (values already rounded to bf16), b: [32]. Nothing is done when
// *done or *skip (the learned term switched off).
__global__ void __launch_bounds__(NET_THREADS) k_net_in(const float2* __restrict__ in, int X, int Y, long P,
		const float* __restrict__ w, const float* __restrict__ b, const float* scale, const double* norm_part,
		int nnorm, bf16* __restrict__ out, const int* done, const int* skip)
{
	__shared__ float sw[NET_C * 18 + NET_C];
	__shared__ double red[32];

	if ((done && *done) || (skip && *skip))
		return;

	for (int i = threadIdx.x; i < NET_C * 18 + NET_C; i += NET_THREADS)
		sw[i] = (i < NET_C * 18) ? w[i] : b[i - NET_C * 18];

	float s = 1.f;

	if (scale) {

		s = *scale;

	} else if (norm_part) {

		const double n2 = sum_partials_d(norm_part, nnorm, red);
		s = (n2 > 0.) ? (float)(1. / sqrt(n2)) : 0.f;
	}

	__syncthreads();

	const long p = (long)blockIdx.x * NET_THREADS + threadIdx.x;

	if (p >= P)
		return;

	const long XY = (long)X * Y;
	const long base = (p / XY) * XY;
	const int y = (int)((p % XY) / X);
	const int x = (int)(p % X);
	float v[18];
#pragma unroll
	for (int tap = 0; tap < 9; tap++) {

		int yy = y + tap / 3 - 1;
		int xx = x + tap % 3 - 1;
		float2 u = make_float2(0.f, 0.f);

		if ((yy >= 0) && (yy < Y) && (xx >= 0) && (xx < X))
			u = in[base + (long)yy * X + xx];

		v[2 * tap] = u.x * s;
		v[2 * tap + 1] = u.y * s;
	}

	// the pixel's 32 channels leave as four 16-byte stores
	uint32_t pk[16];
#pragma unroll
	for (int co = 0; co < NET_C; co += 2) {

		float a0 = sw[NET_C * 18 + co];
		float a1 = sw[NET_C * 18 + co + 1];
#pragma unroll
		for (int k = 0; k < 18; k++) {

			a0 = fmaf(sw[co * 18 + k], v[k], a0);
			a1 = fmaf(sw[(co + 1) * 18 + k], v[k], a1);
		}

		const bf162 h = __floats2bfloat162_rn(fmaxf(a0, 0.f), fmaxf(a1, 0.f));
		pk[co / 2] = *(const uint32_t*)&h;
	}

	uint4* o = (uint4*)(out + p * NET_C);
#pragma unroll
	for (int q = 0; q < 4; q++)
		o[q] = make_uint4(pk[4 * q], pk[4 * q + 1], pk[4 * q + 2], pk[4 * q + 3]);
}

// sum over the 3x3 neighbourhood of a 32-channel bf16 activation with
// weights w[co][tap][ci] (float), co in {0, 1}
__device__ __forceinline__ float2 net_out_pixel(const bf16* __restrict__ act, long base, int x, int y, int X, int Y,
		const float* sw)
{
	float o0 = 0.f, o1 = 0.f;
#pragma unroll 1
	for (int tap = 0; tap < 9; tap++) {

		int yy = y + tap / 3 - 1;
		int xx = x + tap % 3 - 1;

		if ((yy < 0) || (yy >= Y) || (xx < 0) || (xx >= X))
			continue;

		const uint4* a = (const uint4*)(act + (base + (long)yy * X + xx) * NET_C);
#pragma unroll
		for (int q = 0; q < 4; q++) {

			uint4 u = a[q];
			const bf162* h = (const bf162*)&u;
#pragma unroll
			for (int j = 0; j < 4; j++) {

				float2 f = __bfloat1622float2(h[j]);
				int ci = q * 8 + 2 * j;
				o0 = fmaf(sw[tap * NET_C + ci], f.x, o0);
				o0 = fmaf(sw[tap * NET_C + ci + 1], f.y, o0);
				o1 = fmaf(sw[9 * NET_C + tap * NET_C + ci], f.x, o1);
				o1 = fmaf(sw[9 * NET_C + tap * NET_C + ci + 1], f.y, o1);
			}
		}
	}

	return make_float2(o0, o1);
}

// Layer 6 (32 -> 2), one thread per pixel:
//   out = zc + s * (conv(act, w) + b)   (zc = 0 if null),
// s = *scale, or sqrt(sum of norm_part) (the norm of zc, from the partials
// of the pass that wrote it), or 1; out = zc when *net_off (the stall
// fallback of the flexible CG). With pdot: per-block partials Re<pdot, out>.
__global__ void __launch_bounds__(NET_THREADS) k_net_out(const bf16* __restrict__ act, int X, int Y, long P,
		const float* __restrict__ w, const float* __restrict__ b, const float* scale, const double* norm_part,
		int nnorm, const float2* zc, float2* out, const float2* __restrict__ pdot, double* __restrict__ dot_part,
		const int* done, const int* net_off)
{
	__shared__ float sw[2 * 9 * NET_C + 2];
	__shared__ double red[32];

	if (done && *done)
		return;

	for (int i = threadIdx.x; i < 2 * 9 * NET_C + 2; i += NET_THREADS)
		sw[i] = (i < 2 * 9 * NET_C) ? w[i] : b[i - 2 * 9 * NET_C];

	const float s = scale ? *scale : (norm_part ? (float)sqrt(sum_partials_d(norm_part, nnorm, red)) : 1.f);
	__syncthreads();

	const long p = (long)blockIdx.x * NET_THREADS + threadIdx.x;
	const bool off = net_off && *net_off;
	double dot = 0.;

	if (p < P) {

		const long XY = (long)X * Y;
		float2 v = zc ? zc[p] : make_float2(0.f, 0.f);

		if (!off) {

			float2 o = net_out_pixel(act, (p / XY) * XY, (int)(p % X), (int)((p % XY) / X), X, Y, sw);
			v.x = fmaf(s, o.x + sw[2 * 9 * NET_C], v.x);
			v.y = fmaf(s, o.y + sw[2 * 9 * NET_C + 1], v.y);
		}

		out[p] = v;

		if (pdot) {

			float2 q = pdot[p];
			dot = (double)q.x * (double)v.x + (double)q.y * (double)v.y;
		}
	}

	if (pdot) {

		double t = block_sum_d(dot, red);

		if (0 == threadIdx.x)
			dot_part[blockIdx.x] = t;
	}
}

// Backward of layer 6 to its input, masked by the ReLU of layer 5:
//   gu5[q][ci] = bf16((act5[q][ci] > 0) * sum_{co, tap} w[co][8 - tap][ci] gout[q + off(tap)][co])
__global__ void __launch_bounds__(NET_THREADS) k_net_out_bwd(const float2* __restrict__ gout, const bf16* __restrict__ act5,
		int X, int Y, long P, const float* __restrict__ w, bf16* __restrict__ gu5)
{
	__shared__ float sw[2 * 9 * NET_C];

	for (int i = threadIdx.x; i < 2 * 9 * NET_C; i += NET_THREADS)
		sw[i] = w[i];

	__syncthreads();

	const long q = (long)blockIdx.x * NET_THREADS + threadIdx.x;

	if (q >= P)
		return;

	const long XY = (long)X * Y;
	const long base = (q / XY) * XY;
	const int y = (int)((q % XY) / X);
	const int x = (int)(q % X);
	float2 gn[9];
#pragma unroll
	for (int tap = 0; tap < 9; tap++) {

		int yy = y + tap / 3 - 1;
		int xx = x + tap % 3 - 1;
		gn[tap] = ((yy >= 0) && (yy < Y) && (xx >= 0) && (xx < X)) ? gout[base + (long)yy * X + xx] : make_float2(0.f, 0.f);
	}

	const bf162* m = (const bf162*)(act5 + q * NET_C);
	bf162* o = (bf162*)(gu5 + q * NET_C);
#pragma unroll 2
	for (int ci = 0; ci < NET_C; ci += 2) {

		float a0 = 0.f, a1 = 0.f;
#pragma unroll
		for (int tap = 0; tap < 9; tap++) {

			int ft = 8 - tap;
			a0 = fmaf(sw[ft * NET_C + ci], gn[tap].x, a0);
			a0 = fmaf(sw[9 * NET_C + ft * NET_C + ci], gn[tap].y, a0);
			a1 = fmaf(sw[ft * NET_C + ci + 1], gn[tap].x, a1);
			a1 = fmaf(sw[9 * NET_C + ft * NET_C + ci + 1], gn[tap].y, a1);
		}

		float2 mk = __bfloat1622float2(m[ci / 2]);
		o[ci / 2] = __floats2bfloat162_rn((mk.x > 0.f) ? a0 : 0.f, (mk.y > 0.f) ? a1 : 0.f);
	}
}

__device__ __forceinline__ float net_load(const bf16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ float net_load(const float* p) { return *p; }

// Weight and bias gradients of a 3x3 layer, per block of a 32 x 8 pixel tile:
//   part[blk][(co * 9 + tap) * CIN + ci] = sum_p g[p][co] a[p + off(tap)][ci]
//   part[blk][COUT * 9 * CIN + co]        = sum_p g[p][co]
// a: [P][CIN], g: [P][COUT] (bf16 or float). grid (ceil(X/32), ceil(Y/8), nimg).
template <int CIN, int COUT, typename AT, typename GT>
__global__ void __launch_bounds__(NET_THREADS) k_wgrad(const AT* __restrict__ a, const GT* __restrict__ g, int X, int Y,
		float* __restrict__ part)
{
	extern __shared__ float wg_smem[];
	float* sa = wg_smem;					// [10][34][CIN]
	float* sg = sa + NET_HALO_Y * NET_HALO_X * CIN;		// [8][32][COUT]
	constexpr int O = COUT * 9 * CIN;

	const int x0 = blockIdx.x * NET_TILE_X;
	const int y0 = blockIdx.y * NET_TILE_Y;
	const long ibase = (long)blockIdx.z * X * Y;

	for (int i = threadIdx.x; i < NET_HALO_Y * NET_HALO_X * CIN; i += NET_THREADS) {

		int ci = i % CIN;
		int pix = i / CIN;
		int gy = y0 + pix / NET_HALO_X - 1;
		int gx = x0 + pix % NET_HALO_X - 1;
		sa[i] = ((gy >= 0) && (gy < Y) && (gx >= 0) && (gx < X)) ? net_load(a + (ibase + (long)gy * X + gx) * CIN + ci) : 0.f;
	}

	for (int i = threadIdx.x; i < NET_TILE_Y * NET_TILE_X * COUT; i += NET_THREADS) {

		int co = i % COUT;
		int pix = i / COUT;
		int gy = y0 + pix / NET_TILE_X;
		int gx = x0 + pix % NET_TILE_X;
		sg[i] = ((gy < Y) && (gx < X)) ? net_load(g + (ibase + (long)gy * X + gx) * COUT + co) : 0.f;
	}

	__syncthreads();

	float* dst = part + (long)(blockIdx.x + gridDim.x * (blockIdx.y + (long)gridDim.y * blockIdx.z)) * (O + COUT);

	for (int o = threadIdx.x; o < O + COUT; o += NET_THREADS) {

		float acc = 0.f;

		if (o < O) {

			const int co = o / (9 * CIN);
			const int tap = (o / CIN) % 9;
			const int ci = o % CIN;
			const int ky = tap / 3;
			const int kx = tap % 3;
#pragma unroll 4
			for (int py = 0; py < NET_TILE_Y; py++)
				for (int px = 0; px < NET_TILE_X; px++)
					acc = fmaf(sg[(py * NET_TILE_X + px) * COUT + co],
						sa[((py + ky) * NET_HALO_X + px + kx) * CIN + ci], acc);

		} else {

			const int co = o - O;

			for (int pix = 0; pix < NET_TILE_Y * NET_TILE_X; pix++)
				acc += sg[pix * COUT + co];
		}

		dst[o] = acc;
	}
}

// grad[o] = sum over blocks of part[blk][o], in block order
__global__ void k_wgrad_reduce(const float* __restrict__ part, long nblk, int O, float* __restrict__ grad)
{
	const int o = blockIdx.x * blockDim.x + threadIdx.x;

	if (o >= O)
		return;

	double acc = 0.;

	for (long k = 0; k < nblk; k++)
		acc += part[k * O + o];

	grad[o] = (float)acc;
}

// gout = c (out - target), loss partials sum |out - target|^2 per block
__global__ void k_net_loss(const float2* __restrict__ out, const float2* __restrict__ target, long P, float c,
		float2* __restrict__ gout, double* __restrict__ loss_part)
{
	__shared__ double red[32];
	double acc = 0.;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < P; i += (long)gridDim.x * blockDim.x) {

		float2 d = make_float2(out[i].x - target[i].x, out[i].y - target[i].y);
		gout[i] = make_float2(c * d.x, c * d.y);
		acc += (double)d.x * d.x + (double)d.y * d.y;
	}

	double t = block_sum_d(acc, red);

	if (0 == threadIdx.x)
		loss_part[blockIdx.x] = t;
}

// Adam (Kingma & Ba, ICLR 2015) on the float32 master parameters
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ gr, float* __restrict__ m, float* __restrict__ v,
		int n, float lr, float b1, float b2, float eps, float c1, float c2)
{
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {

		float gi = gr[i];
		float mi = b1 * m[i] + (1.f - b1) * gi;
		float vi = b2 * v[i] + (1.f - b2) * gi * gi;
		m[i] = mi;
		v[i] = vi;
		p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
	}
}

// Working copies of the parameters: float values rounded to bf16 (all
// weights; biases stay float) and, for layers 2-5, bf16 forward weights
// [co][tap][ci] and transposed tap-flipped weights [ci][8 - tap][co].
__global__ void k_net_pack(const float* __restrict__ p, float* __restrict__ pr, bf16* __restrict__ wf, bf16* __restrict__ wt)
{
	const int n = NetLayout::total();

	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {

		int l = 0;

		while ((l < 5) && (i >= NetLayout::woff(l + 1)))
			l++;

		const int r = i - NetLayout::woff(l);
		const bool weight = (r < NetLayout::wsize(l));
		bf16 h = __float2bfloat16_rn(p[i]);
		pr[i] = weight ? __bfloat162float(h) : p[i];

		if (weight && (l >= 1) && (l <= 4)) {

			const int co = r / 288;
			const int tap = (r / 32) % 9;
			const int ci = r % 32;
			wf[(l - 1) * 9216 + r] = h;
			wt[(l - 1) * 9216 + (ci * 9 + (8 - tap)) * 32 + co] = h;
		}
	}
}

} // namespace bn
