// Binned Kaiser-Bessel gridding and degridding through shared-memory tiles.
//
// Plan time: every sample gets the bin (tile of BS^d cells of the oversampled
// grid) holding its centre 2k + N per axis; a stable radix sort orders the
// samples by bin, and bins are cut into sub-blocks of at most SUB samples
// (dense bins at the k-space centre become several sub-blocks, so the work
// is balanced). The sorted trajectory is stored as float4 (coalesced loads).
//
// Degridding (gather): a block takes one sub-block, loads its bin's tile plus
// a halo of HALO cells per side for a chunk of coils into shared memory
// (coalesced rows), then every sample gathers its taps from the tile.
// Gridding (scatter): a block accumulates its samples' taps into a zeroed
// shared-memory tile with shared-memory atomics and flushes the touched cells
// to the grid with one global float2 atomic each, instead of one global atomic
// per tap.
//
// Taps and weights are those of axis_taps (bit-identical to the reference's,
// src/noncart/grid.c:403-465); only the cell index changes from the DFT-order
// grid index to the tile-local index of the same cell.
#pragma once

#include <cuda_runtime.h>

#include "nufft_kernels.cuh"

namespace bn {

enum { BIN_HALO = 4, BIN_SUB = 512, BIN_THREADS = 256 };

struct BinGeom {

	int bs[3];	// bin size per axis (1 for singleton axes)
	int nb[3];	// bins per axis
	int tile[3];	// tile extent per axis (bs + 2 * halo, or 1)
	long ncells;	// tile cells
};

// Taps of one axis relative to a tile origin (centred 2N index of the tile's
// first cell). Same taps / weights as axis_taps; cell = tile-local index.
__device__ __forceinline__ void axis_taps_local(float k, int N, float hw, int periodic, const float* kb,
		int origin, int extent, AxisTaps& t)
{
	t.n = 0;

	if (1 == N) {

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
			int local = 2 * w + s - origin;

			if (periodic)	// the tap may sit one period away from the tile
				local = ((local % L) + L) % L;

			if ((local < 0) || (local >= extent))
				continue;	// cannot happen for a sample of this bin

			t.cell[t.n] = local;
			t.w[t.n] = val;
			t.n++;
		}
	}
}

// centred 2N position of a sample along an axis -> bin index
__device__ __forceinline__ int bin_of(float k, int N, int bs, int nb, int periodic)
{
	if (1 == N)
		return 0;

	float p = 2.f * k + (float)N;

	if (periodic) {

		float L = 2.f * N;
		p = p - L * floorf(p / L);
	}

	int b = (int)floorf(p / (float)bs);
	return min(max(b, 0), nb - 1);
}

// key = bin id of sample m, value = m
__global__ void k_bin_keys(const float4* __restrict__ traj, long M, GridGeom g, BinGeom bg,
		unsigned* __restrict__ keys, int* __restrict__ vals, int* __restrict__ counts)
{
	for (long m = (long)blockIdx.x * blockDim.x + threadIdx.x; m < M; m += (long)gridDim.x * blockDim.x) {

		float4 k = traj[m];
		int bx = bin_of(k.x, g.N[0], bg.bs[0], bg.nb[0], g.periodic);
		int by = bin_of(k.y, g.N[1], bg.bs[1], bg.nb[1], g.periodic);
		int bz = bin_of(k.z, g.N[2], bg.bs[2], bg.nb[2], g.periodic);
		unsigned key = (unsigned)(bx + bg.nb[0] * (by + bg.nb[1] * bz));
		keys[m] = key;
		vals[m] = (int)m;
		atomicAdd(&counts[key], 1);
	}
}

// nsub[b] = ceil(count_b / SUB), nsub[nbins] = 0
__global__ void k_bin_nsub(const int* __restrict__ bin_start, int nbins, int* __restrict__ nsub)
{
	for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= nbins; b += gridDim.x * blockDim.x)
		nsub[b] = (b < nbins) ? (bin_start[b + 1] - bin_start[b] + BIN_SUB - 1) / BIN_SUB : 0;
}

// sub-block table: for bin b with n samples starting at bin_start[b],
// ceil(n / SUB) entries (bin, first sample, count) starting at sub_start[b]
__global__ void k_sub_fill(const int* __restrict__ bin_start, const int* __restrict__ sub_start, int nbins,
		int* __restrict__ sub_bin, int* __restrict__ sub_first, int* __restrict__ sub_count)
{
	for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbins; b += gridDim.x * blockDim.x) {

		int n = bin_start[b + 1] - bin_start[b];
		int s0 = sub_start[b];

		for (int j = 0; j * BIN_SUB < n; j++) {

			sub_bin[s0 + j] = b;
			sub_first[s0 + j] = bin_start[b] + j * BIN_SUB;
			sub_count[s0 + j] = min(BIN_SUB, n - j * BIN_SUB);
		}
	}
}

__global__ void k_gather_traj(float4* __restrict__ dst, const float4* __restrict__ src, const int* __restrict__ perm, long M)
{
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (long)gridDim.x * blockDim.x)
		dst[i] = src[perm[i]];
}

struct TileOrigin {

	int o[3];	// centred 2N index of the tile's first cell per axis
};

__device__ __forceinline__ TileOrigin tile_origin(int bin, const BinGeom& bg, const GridGeom& g)
{
	TileOrigin t;
	int bx = bin % bg.nb[0];
	int by = (bin / bg.nb[0]) % bg.nb[1];
	int bz = bin / (bg.nb[0] * bg.nb[1]);
	t.o[0] = (g.N[0] > 1) ? bx * bg.bs[0] - BIN_HALO : 0;
	t.o[1] = (g.N[1] > 1) ? by * bg.bs[1] - BIN_HALO : 0;
	t.o[2] = (g.N[2] > 1) ? bz * bg.bs[2] - BIN_HALO : 0;
	return t;
}

// grid (DFT order) index of tile cell (lx, ly, lz), or -1 outside a
// non-periodic grid
__device__ __forceinline__ long tile_to_grid(int lx, int ly, int lz, const TileOrigin& to, const GridGeom& g)
{
	int l[3] = { lx, ly, lz };
	long idx = 0;
	long stride = 1;

	for (int a = 0; a < 3; a++) {

		int j = 0;

		if (g.N[a] > 1) {

			const int L = g.G[a];
			j = to.o[a] + l[a];

			if ((j < 0) || (j >= L)) {

				if (!g.periodic)
					return -1;

				j = ((j % L) + L) % L;
			}

			j += g.N[a];

			if (j >= L)
				j -= L;
		}

		idx += j * stride;
		stride *= g.G[a];
	}

	return idx;
}

// Degridding: ksp[perm[i] + M*c] for the samples of each sub-block, coils in
// chunks of cc tiles held in shared memory at once.
__global__ void __launch_bounds__(BIN_THREADS) k_degrid_binned(const float4* __restrict__ traj_sorted,
		const int* __restrict__ perm, long M, GridGeom g, BinGeom bg,
		const int* __restrict__ sub_bin, const int* __restrict__ sub_first, const int* __restrict__ sub_count,
		int C, int cc, const float2* __restrict__ grid, float2* __restrict__ ksp, const float* __restrict__ kbg)
{
	extern __shared__ float2 tiles[];	// [cc][ncells]
	__shared__ float kb[KB_TABLE_N + 1];

	for (int i = threadIdx.x; i <= KB_TABLE_N; i += blockDim.x)
		kb[i] = kbg[i];

	const int sb = blockIdx.x;
	const int bin = sub_bin[sb];
	const int first = sub_first[sb];
	const int count = sub_count[sb];
	const TileOrigin to = tile_origin(bin, bg, g);
	const int tx = bg.tile[0], ty = bg.tile[1];

	for (int c0 = 0; c0 < C; c0 += cc) {

		const int cn = min(cc, C - c0);

		__syncthreads();	// previous chunk's readers are done

		for (long t = threadIdx.x; t < bg.ncells * cn; t += blockDim.x) {

			int c = (int)(t / bg.ncells);
			long cell = t - (long)c * bg.ncells;
			int lx = (int)(cell % tx);
			int ly = (int)((cell / tx) % ty);
			int lz = (int)(cell / ((long)tx * ty));
			long gi = tile_to_grid(lx, ly, lz, to, g);
			tiles[(long)c * bg.ncells + cell] = (gi >= 0) ? grid[gi + g.gsz * (c0 + c)] : make_float2(0.f, 0.f);
		}

		__syncthreads();

		for (int i = threadIdx.x; i < count; i += blockDim.x) {

			float4 k = traj_sorted[first + i];
			AxisTaps ax, ay, az;
			axis_taps_local(k.x, g.N[0], g.hw, g.periodic, kb, to.o[0], bg.tile[0], ax);
			axis_taps_local(k.y, g.N[1], g.hw, g.periodic, kb, to.o[1], bg.tile[1], ay);
			axis_taps_local(k.z, g.N[2], g.hw, g.periodic, kb, to.o[2], bg.tile[2], az);
			const long m = perm[first + i];

			for (int c = 0; c < cn; c++) {

				const float2* tl = tiles + (long)c * bg.ncells;
				float2 acc = make_float2(0.f, 0.f);

				for (int a = 0; a < az.n; a++) {

					float dz = az.w[a];
					int oz = az.cell[a] * ty;

					for (int b = 0; b < ay.n; b++) {

						float dzy = __fmul_rn(dz, ay.w[b]);
						int oy = (oz + ay.cell[b]) * tx;

						for (int e = 0; e < ax.n; e++) {

							float d = __fmul_rn(dzy, ax.w[e]);
							float2 v = tl[oy + ax.cell[e]];
							acc.x = fmaf(v.x, d, acc.x);
							acc.y = fmaf(v.y, d, acc.y);
						}
					}
				}

				ksp[m + M * (c0 + c)] = acc;
			}
		}
	}
}

// Gridding: per sub-block, shared-memory accumulation then one global atomic
// per touched tile cell. The grid must be zeroed.
__global__ void __launch_bounds__(BIN_THREADS) k_grid_binned(const float4* __restrict__ traj_sorted,
		const int* __restrict__ perm, long M, GridGeom g, BinGeom bg,
		const int* __restrict__ sub_bin, const int* __restrict__ sub_first, const int* __restrict__ sub_count,
		int C, int cc, const float2* __restrict__ ksp, float2* __restrict__ grid, const float* __restrict__ kbg)
{
	extern __shared__ float2 tiles[];	// [cc][ncells]
	__shared__ float kb[KB_TABLE_N + 1];

	for (int i = threadIdx.x; i <= KB_TABLE_N; i += blockDim.x)
		kb[i] = kbg[i];

	const int sb = blockIdx.x;
	const int bin = sub_bin[sb];
	const int first = sub_first[sb];
	const int count = sub_count[sb];
	const TileOrigin to = tile_origin(bin, bg, g);
	const int tx = bg.tile[0], ty = bg.tile[1];

	for (int c0 = 0; c0 < C; c0 += cc) {

		const int cn = min(cc, C - c0);

		__syncthreads();

		for (long t = threadIdx.x; t < bg.ncells * cn; t += blockDim.x)
			tiles[t] = make_float2(0.f, 0.f);

		__syncthreads();

		for (int i = threadIdx.x; i < count; i += blockDim.x) {

			float4 k = traj_sorted[first + i];
			AxisTaps ax, ay, az;
			axis_taps_local(k.x, g.N[0], g.hw, g.periodic, kb, to.o[0], bg.tile[0], ax);
			axis_taps_local(k.y, g.N[1], g.hw, g.periodic, kb, to.o[1], bg.tile[1], ay);
			axis_taps_local(k.z, g.N[2], g.hw, g.periodic, kb, to.o[2], bg.tile[2], az);
			const long m = perm[first + i];

			for (int c = 0; c < cn; c++) {

				float2 val = ksp[m + M * (c0 + c)];

				if ((0.f == val.x) && (0.f == val.y))
					continue;

				float* tl = (float*)(tiles + (long)c * bg.ncells);

				for (int a = 0; a < az.n; a++) {

					float dz = az.w[a];
					int oz = az.cell[a] * ty;

					for (int b = 0; b < ay.n; b++) {

						float dzy = __fmul_rn(dz, ay.w[b]);
						int oy = (oz + ay.cell[b]) * tx;

						for (int e = 0; e < ax.n; e++) {

							float d = __fmul_rn(dzy, ax.w[e]);
							int cell = oy + ax.cell[e];
							atomicAdd(&tl[2 * cell + 0], val.x * d);
							atomicAdd(&tl[2 * cell + 1], val.y * d);
						}
					}
				}
			}
		}

		__syncthreads();

		for (long t = threadIdx.x; t < bg.ncells * cn; t += blockDim.x) {

			float2 v = tiles[t];

			if ((0.f == v.x) && (0.f == v.y))
				continue;

			int c = (int)(t / bg.ncells);
			long cell = t - (long)c * bg.ncells;
			int lx = (int)(cell % tx);
			int ly = (int)((cell / tx) % ty);
			int lz = (int)(cell / ((long)tx * ty));
			long gi = tile_to_grid(lx, ly, lz, to, g);

			if (gi >= 0)
				atomicAdd(&grid[gi + g.gsz * (c0 + c)], v);
		}
	}
}

} // namespace bn
