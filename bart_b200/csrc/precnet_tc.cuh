// 32 -> 32 channel 3x3 convolution of the learned preconditioner on the
// fifth-generation tensor cores: TMA tile loads into shared memory,
// tcgen05.mma with the accumulator in tensor memory, tcgen05.ld epilogue.
//
// Implicit GEMM. A work tile is R image rows of 128 pixels (x0 .. x0 + 127
// of rows y0 .. y0 + R - 1) for all 32 output channels. Per row the product
// is D[128 px][32 cout] = sum over 9 taps and 2 halves of 16 input channels
// of A_tap[128 px][16 cin] B_tap[16 cin][32 cout]: 18 MMAs of M = 128,
// N = 32, K = 16 (bf16 inputs, float32 accumulation), issued by one thread;
// R accumulators of 32 TMEM columns.
//
// Operands use the canonical K-major layout without swizzle: 8-row x 16-byte
// core matrices (rows 16 B apart), 8-row groups SBO = 128 B apart, the two
// 8-element K chunks of one MMA LBO apart.
//  * A: the halo tile (R + 2 rows x 130 pixels) as four channel planes,
//    plane j = channels 8j .. 8j + 7 of every halo pixel, 16 B per pixel.
//    Each plane is one TMA load of a {8 channels, 130, R + 2, 1} box of the
//    NHWC activation tensor [nimg][Y][X][32] (4D tensor map); out-of-image
//    pixels are zero-filled by the TMA unit. The A operand of tap (ky, kx)
//    for output row r is the same planes started (r + ky) * 130 + kx pixels
//    in: one descriptor per MMA, no data movement.
//  * B: the weights prepacked as 36 planes of 32 rows x 16 B (plane =
//    tap * 4 + cin / 8, row = cout), one bulk copy of 18 KB per block.
// Blocks are persistent: each loads the weights once and walks the tiles
// blockIdx.x, + gridDim.x, ...; several blocks share an SM, so one block's
// loads overlap another's MMAs and epilogue.
//
// Epilogue: warp w reads TMEM lanes 32w .. 32w + 31 (= pixels), 32 columns
// (= output channels) per thread; MODE 0 adds the bias and applies the ReLU,
// MODE 1 applies the ReLU mask of the layer below (data gradient with the
// transposed, tap-flipped weights); bf16 NHWC stores, 64 B per pixel.
//
// Every wait is bounded: past TC_SPIN_LIMIT polls the block records the
// failure in *status, waits (bounded again) for what it has in flight,
// releases its tensor memory and leaves.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "precnet.cuh"

namespace bn {

enum { TC_M = 128, TC_HX = TC_M + 2, TC_SPIN_LIMIT = 1 << 22, TC_W_BYTES = 36 * 512 };

// bytes of one A channel plane
__host__ __device__ constexpr uint32_t conv_tc_plane(int R) { return (uint32_t)(R + 2) * TC_HX * 16; }

// shared-memory bytes: A planes, B planes, two mbarriers and the TMEM slot
__host__ __device__ constexpr size_t conv_tc_smem(int R) { return (size_t)4 * conv_tc_plane(R) + TC_W_BYTES + 32; }

// TMEM columns: R accumulators of 32 columns, a power of two >= 32
__host__ __device__ constexpr uint32_t conv_tc_cols(int R)
{
	return (R * 32 <= 32) ? 32 : (R * 32 <= 64) ? 64 : (R * 32 <= 128) ? 128 : 256;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
	return (uint32_t)__cvta_generic_to_shared(p);
}

// K-major, no swizzle: start, LBO (K-chunk stride), SBO (8-row group stride),
// descriptor version 1
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
	return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16)
		| ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// kind::f16 instruction descriptor: D float32 (bits 4-5), A and B bf16
// (bits 7-9, 10-12), both K-major, N >> 3 (bits 17-22), M >> 4 (bits 24-28)
constexpr uint32_t CONV_TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
	asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
		:: "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
	uint32_t ok;
	asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
		: "=r"(ok) : "r"(bar), "r"(parity) : "memory");
	return 0 != ok;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity)
{
	for (int it = 0; it < TC_SPIN_LIMIT; it++)
		if (mbar_try_wait(bar, parity))
			return true;

	return false;
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" :: "r"(bar), "r"(bytes) : "memory");
}

// 4D tiled TMA load (no multicast) of the tensor map's box at (c0, c1, c2, c3)
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, uint32_t bar)
{
	asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n"
		:: "r"(dst), "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar) : "memory");
}

// plain bulk copy global -> shared (16-byte aligned, size a multiple of 16)
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
		:: "r"(dst), "l"((uint64_t)src), "r"(bytes), "r"(bar) : "memory");
}

// 32 consecutive TMEM columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
	uint32_t r[32];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
		"{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
		"%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
		: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
		  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
		  "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
		  "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
		: "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
	for (int i = 0; i < 32; i++)
		v[i] = __uint_as_float(r[i]);
}

// Weights of the four 32 -> 32 layers, [layer][cout][tap][cin] (bf16), into
// the B-plane order [layer][tap * 4 + cin / 8][cout][cin % 8].
__global__ void k_net_pack_tc(const bf16* __restrict__ w, bf16* __restrict__ wp)
{
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 4 * 9216; i += gridDim.x * blockDim.x) {

		const int l = i / 9216, r = i % 9216;
		const int co = r / 288, k = r % 288;	// k = tap * 32 + cin
		wp[l * 9216 + (k / 8) * 256 + co * 8 + (k % 8)] = w[i];
	}
}

// in: the tensor map of the input activations [nimg][Y][X][32] bf16 with a
// box of {8, 130, R + 2, 1}; wp: one layer's prepacked weights; tiles =
// ceil(X / 128) * ceil(Y / R) * nimg; 128 threads per block.
template <int MODE, int R>
__global__ void __launch_bounds__(128) k_conv32_tc(const __grid_constant__ CUtensorMap in, const bf16* __restrict__ wp,
		const float* __restrict__ bias, const bf16* __restrict__ mask, bf16* __restrict__ out, int X, int Y,
		int nimg, const int* done, const int* skip, int* status)
{
	constexpr uint32_t PLANE = conv_tc_plane(R);
	constexpr uint32_t NCOL = conv_tc_cols(R);
	extern __shared__ __align__(128) unsigned char tc_smem[];
	unsigned char* sA = tc_smem;				// 4 planes
	unsigned char* sB = tc_smem + 4 * PLANE;		// 36 planes of 512 B
	uint64_t* bars = (uint64_t*)(sB + TC_W_BYTES);		// [0] loads, [1] MMAs
	uint32_t* tslot = (uint32_t*)(bars + 2);

	if ((done && *done) || (skip && *skip))
		return;

	const int tid = threadIdx.x;
	const int warp = tid >> 5;
	const int tx = (X + TC_M - 1) / TC_M, ty = (Y + R - 1) / R;
	const long ntiles = (long)tx * ty * nimg;

	if ((long)blockIdx.x >= ntiles)
		return;

	const uint32_t lbar = smem_u32(&bars[0]), mbar = smem_u32(&bars[1]);

	if (0 == warp) {	// tensor memory for the R accumulators

		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
			:: "r"(smem_u32(tslot)), "r"(NCOL) : "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
	}

	if (0 == tid) {

		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" :: "r"(lbar) : "memory");
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" :: "r"(mbar) : "memory");
		asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
		asm volatile("prefetch.tensormap [%0];\n" :: "l"((uint64_t)&in) : "memory");
	}

	asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");

	const uint32_t tmem = *tslot;
	const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
	int failed = 0;
	uint32_t phase = 0;	// uses of each barrier so far (parity of the next wait)
	bool mma_pending = false, load_pending = false;

	for (long t = blockIdx.x; t < ntiles; t += gridDim.x, phase ^= 1u) {

		const int img = (int)(t / ((long)tx * ty));
		const int rem = (int)(t % ((long)tx * ty));
		const int x0 = (rem % tx) * TC_M;
		const int y0 = (rem / tx) * R;

		if (0 == tid) {	// halo planes (and the weights with the first tile)

			const bool first = ((long)blockIdx.x == t);
			mbar_expect_tx(lbar, 4 * PLANE + (first ? TC_W_BYTES : 0));

			if (first)
				bulk_load(b0, wp, TC_W_BYTES, lbar);

			for (int j = 0; j < 4; j++)
				tma_load_4d(a0 + j * PLANE, &in, 8 * j, x0 - 1, y0 - 1, img, lbar);
		}

		load_pending = true;
		bool ok = mbar_wait_bounded(lbar, phase);

		if (!__syncthreads_and(ok ? 1 : 0)) {

			failed = 1;
			break;
		}

		load_pending = false;

		if (0 == tid) {

			asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll 1
			for (int r = 0; r < R; r++) {
#pragma unroll 1
				for (int tap = 0; tap < 9; tap++) {

					const int ky = tap / 3, kx = tap % 3;
					const uint32_t shift = (uint32_t)(((r + ky) * TC_HX + kx) * 16);
#pragma unroll
					for (int h = 0; h < 2; h++) {

						const uint64_t da = umma_desc(a0 + 2 * h * PLANE + shift, PLANE, 128);
						const uint64_t db = umma_desc(b0 + (tap * 4 + 2 * h) * 512, 512, 128);
						umma_f16(tmem + r * 32, da, db, CONV_TC_IDESC, (tap | h) ? 1u : 0u);
					}
				}
			}

			asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
				:: "r"(mbar) : "memory");
		}

		mma_pending = true;
		ok = mbar_wait_bounded(mbar, phase);

		if (!__syncthreads_and(ok ? 1 : 0)) {

			failed = 1;
			break;
		}

		mma_pending = false;
		asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
		const int px = x0 + tid;	// this thread's pixel (TMEM lane = tid)
#pragma unroll 1
		for (int r = 0; r < R; r++) {

			float v[32];
			tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + r * 32, v);
			const int gy = y0 + r;

			if ((px >= X) || (gy >= Y))
				continue;

			const long o = (((long)img * Y + gy) * X + px) * NET_C;
			uint32_t pk[16];
#pragma unroll
			for (int c = 0; c < 32; c += 2) {

				float v0 = v[c], v1 = v[c + 1];

				if (0 == MODE) {

					v0 = fmaxf(v0 + bias[c], 0.f);
					v1 = fmaxf(v1 + bias[c + 1], 0.f);

				} else {

					const bf162 m = *(const bf162*)(mask + o + c);
					v0 = (__bfloat162float(m.x) > 0.f) ? v0 : 0.f;
					v1 = (__bfloat162float(m.y) > 0.f) ? v1 : 0.f;
				}

				const bf162 b2 = __floats2bfloat162_rn(v0, v1);
				pk[c / 2] = *(const uint32_t*)&b2;
			}
#pragma unroll
			for (int q = 0; q < 4; q++)
				((uint4*)(out + o))[q] = make_uint4(pk[4 * q], pk[4 * q + 1], pk[4 * q + 2], pk[4 * q + 3]);
		}

		// all TMEM reads done before the next tile's MMAs overwrite the accumulators
		asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
		__syncthreads();
		asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
	}

	if (failed) {

		if (0 == tid)
			atomicExch(status, 1);

		// what is still in flight may complete late: wait for it (bounded)
		if (load_pending)
			mbar_wait_bounded(lbar, phase);

		if (mma_pending)
			mbar_wait_bounded(mbar, phase);
	}

	asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
	__syncthreads();

	if (0 == warp)
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" :: "r"(tmem), "r"(NCOL) : "memory");
}

} // namespace bn
