// Binned Kaiser-Bessel gridding and degridding through shared-memory tiles.
//
// Plan time: every sample gets the bin (tile of BS^d cells of the oversampled
// grid) holding its centre 2k + N per axis; a stable radix sort orders the
// samples by bin, and bins are cut into sub-blocks of at most SUB samples
// (dense bins at the k-space centre become several sub-blocks, so the work
// is balanced). The sorted trajectory is stored as float4 (coalesced loads).
//
// Degridding (gather): one thread per sample in bin order; neighbouring
// threads read overlapping taps, so the gathers hit L1, and the weights are
// computed once per sample for all coils.
// Gridding (scatter), default: one thread per sample in bin order with one
// global float2 atomic per tap (bin order keeps a block's atomics within a
// few L2 lines). Alternative (BNUFFT_GRIDDING=tiles): a block takes one
// sub-block, accumulates its samples' taps into a zeroed shared-memory tile
// (bin plus HALO cells per side, a chunk of coils) with shared-memory atomics
// and flushes touched cells with one global atomic each; on B200 it measured
// slower for radial and kooshball data.
//
// Taps and weights are those of axis_taps (bit-identical to the reference's,
// src/noncart/grid.c:403-465); only the cell index changes from the DFT-order
// grid index to the tile-local index of the same cell.
#pragma once

#include <climits>
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

// nsub[b] = ceil(count_b / sub), nsub[nbins] = 0
__global__ void k_bin_nsub(const int* __restrict__ bin_start, int nbins, int sub, int* __restrict__ nsub)
{
	for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= nbins; b += gridDim.x * blockDim.x)
		nsub[b] = (b < nbins) ? (bin_start[b + 1] - bin_start[b] + sub - 1) / sub : 0;
}

// sub-block table: for bin b with n samples starting at bin_start[b],
// ceil(n / sub) entries (bin, first sample, count) starting at sub_start[b]
__global__ void k_sub_fill(const int* __restrict__ bin_start, const int* __restrict__ sub_start, int nbins, int sub,
		int* __restrict__ sub_bin, int* __restrict__ sub_first, int* __restrict__ sub_count)
{
	for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbins; b += gridDim.x * blockDim.x) {

		int n = bin_start[b + 1] - bin_start[b];
		int s0 = sub_start[b];

		for (int j = 0; j * sub < n; j++) {

			sub_bin[s0 + j] = b;
			sub_first[s0 + j] = bin_start[b] + j * sub;
			sub_count[s0 + j] = min(sub, n - j * sub);
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

// Width-6 fast path ------------------------------------------------------------
//
// For the default kernel width 6 (hw = 3 on the N-grid) each sub-grid has
// exactly three taps with weight: the window [pos - 1.5, pos + 1.5] holds
// three integers, or four when pos - 1.5 is an integer, and then both end
// taps sit at |t - pos| = 1.5 where the table is exactly 0 (kb(0.5) = 0,
// src/noncart/grid.c:75-76); the lower one is dropped. Taps clipped by a
// non-periodic grid keep weight 0 and a harmless cell index. The fixed trip
// count lets every tap loop unroll into registers.
struct Taps6 {

	int cell[6];
	float w[6];
};

// MODE 0: cell = DFT-order grid index; MODE 1: cell = tile-local index
template <int MODE>
__device__ __forceinline__ void axis_taps6(float k, int N, int periodic, const float* kb, int origin, Taps6& t)
{
	if (1 == N) {
#pragma unroll
		for (int q = 0; q < 6; q++) {

			t.cell[q] = 0;
			t.w[q] = (0 == q) ? kb_lookup(kb, 0.f) : 0.f;
		}

		return;
	}

	const int L = 2 * N;
	const float half = (float)(N / 2);

#pragma unroll
	for (int s = 0; s < 2; s++) {

		float pos = __fadd_rn(__fadd_rn(k, s ? -0.5f : -0.0f), half);
		double lo = (double)pos - 1.5;
		int sti = (int)ceil(lo);

		if ((double)sti == lo)
			sti += 1;

#pragma unroll
		for (int q = 0; q < 3; q++) {

			int w = sti + q;
			float frac = fabsf(__fsub_rn((float)w, pos));
			float val = kb_lookup(kb, __fdiv_rn(frac, 3.0f));
			bool valid = periodic || ((w >= 0) && (w <= N - 1));
			int cell;

			if (0 == MODE) {

				int wm = periodic ? (((w % N) + N) % N) : min(max(w, 0), N - 1);
				cell = 2 * wm + s + N;

				if (cell >= L)
					cell -= L;

			} else {

				cell = 2 * w + s - origin;

				if (periodic)
					cell = ((cell % L) + L) % L;

				cell = max(cell, 0);	// clipped taps (weight 0) may fall left of the tile
			}

			t.cell[3 * s + q] = cell;
			t.w[3 * s + q] = valid ? val : 0.f;
		}
	}
}

// Degridding, width 6: one thread per sample in bin order (coalesced float4
// trajectory loads, neighbouring threads share taps in L1), weights computed
// once and reused for every coil. TZ = 6 for 3D, 1 for 2D.
template <int TZ>
__global__ void __launch_bounds__(BIN_THREADS, 2) k_degrid6(const float4* __restrict__ traj_sorted,
		const int* __restrict__ perm, long M, GridGeom g, int C,
		const float2* __restrict__ grid, float2* __restrict__ ksp, const float* __restrict__ kbg)
{
	__shared__ float kb[KB_TABLE_N + 1];

	for (int i = threadIdx.x; i <= KB_TABLE_N; i += blockDim.x)
		kb[i] = kbg[i];

	__syncthreads();

	long i = (long)blockIdx.x * blockDim.x + threadIdx.x;

	if (i >= M)
		return;

	float4 k = traj_sorted[i];
	Taps6 tx, ty, tz;
	axis_taps6<0>(k.x, g.N[0], g.periodic, kb, 0, tx);
	axis_taps6<0>(k.y, g.N[1], g.periodic, kb, 0, ty);
	axis_taps6<0>(k.z, g.N[2], g.periodic, kb, 0, tz);
	const long m = perm[i];

	// the x taps as an 8-cell window from an even cell: each (z, y) row is
	// read with 4 float4 loads instead of 6 float2 gathers (the gather is
	// bound by L1 requests); windows that wrap around the row read per tap
	int lo = INT_MAX, hi = INT_MIN;
#pragma unroll
	for (int e = 0; e < 6; e++) {

		if (0.f != tx.w[e]) {

			lo = min(lo, tx.cell[e]);
			hi = max(hi, tx.cell[e]);
		}
	}

	const int base = lo & ~1;
	const bool vec = (lo <= hi) && (hi - base < 8);
	float wx8[8];
#pragma unroll
	for (int j = 0; j < 8; j++) {

		float w = 0.f;	// taps with weight only (see k_grid6_atomic)
#pragma unroll
		for (int e = 0; e < 6; e++)
			w = ((0.f != tx.w[e]) && (tx.cell[e] == base + j)) ? tx.w[e] : w;

		wx8[j] = vec ? w : 0.f;
	}

	for (int c = 0; c < C; c++) {

		const float2* gc = grid + g.gsz * c;
		float2 acc = make_float2(0.f, 0.f);
#pragma unroll 1
		for (int a = 0; a < TZ; a++) {

			float dz = tz.w[a];
			long oz = (long)tz.cell[a] * g.G[1];
#pragma unroll
			for (int b = 0; b < 6; b++) {

				float dzy = __fmul_rn(dz, ty.w[b]);
				long oy = (oz + ty.cell[b]) * g.G[0];

				if (vec) {
#pragma unroll
					for (int q = 0; q < 4; q++) {

						// slots past the last tap hold no weight and are not
						// read (the window may pass the end of the row)
						if ((0.f == wx8[2 * q]) && (0.f == wx8[2 * q + 1]))
							continue;

						float d0 = __fmul_rn(dzy, wx8[2 * q]);
						float d1 = __fmul_rn(dzy, wx8[2 * q + 1]);
						float4 v = *(const float4*)(gc + oy + base + 2 * q);
						acc.x = fmaf(v.x, d0, acc.x);
						acc.y = fmaf(v.y, d0, acc.y);
						acc.x = fmaf(v.z, d1, acc.x);
						acc.y = fmaf(v.w, d1, acc.y);
					}

				} else {
#pragma unroll
					for (int e = 0; e < 6; e++) {

						float d = __fmul_rn(dzy, tx.w[e]);
						float2 v = gc[oy + tx.cell[e]];
						acc.x = fmaf(v.x, d, acc.x);
						acc.y = fmaf(v.y, d, acc.y);
					}
				}
			}
		}

		ksp[m + M * c] = acc;
	}
}

// Gridding, width 6: per sub-block, accumulate into shared-memory tiles of cc
// coils with shared-memory atomics, then flush touched cells with one global
// float2 atomic each. The grid must be zeroed.
template <int TZ>
__global__ void __launch_bounds__(BIN_THREADS, 2) k_grid6_binned(const float4* __restrict__ traj_sorted,
		const int* __restrict__ perm, long M, GridGeom g, BinGeom bg,
		const int* __restrict__ sub_bin, const int* __restrict__ sub_first, const int* __restrict__ sub_count,
		const int* __restrict__ nsub_dev, int C, int cc, const float2* __restrict__ ksp, float2* __restrict__ grid,
		const float* __restrict__ kbg)
{
	extern __shared__ float2 tiles[];	// [cc][ncells]
	__shared__ float kb[KB_TABLE_N + 1];

	const int sb = blockIdx.x;

	if (sb >= *nsub_dev)
		return;

	for (int i = threadIdx.x; i <= KB_TABLE_N; i += blockDim.x)
		kb[i] = kbg[i];

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

		// lanes of a warp take samples 8 apart in bin order: neighbouring
		// samples of a trajectory share taps, so this spreads the
		// shared-memory atomics of one instruction over distinct cells
		const int per = (count + blockDim.x - 1) / blockDim.x;

		for (int r = 0; r < per; r++) {

			int t = threadIdx.x + r * blockDim.x;
			int i = (t % 32) * 8 + (t / 32) % 8 + (t / 256) * 256;

			if (i >= count)
				continue;

			float4 k = traj_sorted[first + i];
			Taps6 ax, ay, az;
			axis_taps6<1>(k.x, g.N[0], g.periodic, kb, to.o[0], ax);
			axis_taps6<1>(k.y, g.N[1], g.periodic, kb, to.o[1], ay);
			axis_taps6<1>(k.z, g.N[2], g.periodic, kb, to.o[2], az);
			const long m = perm[first + i];

			for (int c = 0; c < cn; c++) {

				float2 val = ksp[m + M * (c0 + c)];

				if ((0.f == val.x) && (0.f == val.y))
					continue;

				float* tl = (float*)(tiles + (long)c * bg.ncells);
#pragma unroll 1
				for (int a = 0; a < TZ; a++) {

					float dz = az.w[a];
					int oz = az.cell[a] * ty;
#pragma unroll
					for (int b = 0; b < 6; b++) {

						float dzy = __fmul_rn(dz, ay.w[b]);
						int oy = (oz + ay.cell[b]) * tx;
#pragma unroll
						for (int e = 0; e < 6; e++) {

							float d = __fmul_rn(dzy, ax.w[e]);

							if (0.f != d) {

								int cell = oy + ax.cell[e];
								atomicAdd(&tl[2 * cell + 0], val.x * d);
								atomicAdd(&tl[2 * cell + 1], val.y * d);
							}
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

// Gridding, width 6, without tiles: one thread per sample in bin order,
// weights computed once for all coils, global atomics. The scatter is bound
// by the L2's atomic-operation rate, which is the same for 8- and 16-byte
// vector atomics: so the six x-taps of a sample (at most 7 consecutive cells
// of a grid row) are laid into an 8-cell window starting at an even cell,
// and each (z, y) row takes up to 4 float4 atomics (two cells each) instead
// of 6 float2 ones. Windows that wrap around the row fall back to one float2
// atomic per tap. Float sums in another order than the per-tap form: the
// result is the same up to rounding (the atomics' order is arbitrary anyway).
template <int TZ>
__global__ void __launch_bounds__(BIN_THREADS, 2) k_grid6_atomic(const float4* __restrict__ traj_sorted,
		const int* __restrict__ perm, long M, GridGeom g, int C,
		const float2* __restrict__ ksp, float2* __restrict__ grid, const float* __restrict__ kbg)
{
	__shared__ float kb[KB_TABLE_N + 1];

	for (int i = threadIdx.x; i <= KB_TABLE_N; i += blockDim.x)
		kb[i] = kbg[i];

	__syncthreads();

	long i = (long)blockIdx.x * blockDim.x + threadIdx.x;

	if (i >= M)
		return;

	float4 k = traj_sorted[i];
	Taps6 tx, ty, tz;
	axis_taps6<0>(k.x, g.N[0], g.periodic, kb, 0, tx);
	axis_taps6<0>(k.y, g.N[1], g.periodic, kb, 0, ty);
	axis_taps6<0>(k.z, g.N[2], g.periodic, kb, 0, tz);
	const long m = perm[i];

	// the x window: taps with weight, their lowest and highest cell
	int lo = INT_MAX, hi = INT_MIN;
#pragma unroll
	for (int e = 0; e < 6; e++) {

		if (0.f != tx.w[e]) {

			lo = min(lo, tx.cell[e]);
			hi = max(hi, tx.cell[e]);
		}
	}

	const int base = lo & ~1;
	const bool vec = (lo <= hi) && (hi - base < 8);
	float wx8[8];
#pragma unroll
	for (int j = 0; j < 8; j++) {

		// only taps with weight: a clipped tap (weight 0) of a non-periodic
		// grid may sit on the same cell as a valid one
		float w = 0.f;
#pragma unroll
		for (int e = 0; e < 6; e++)
			w = ((0.f != tx.w[e]) && (tx.cell[e] == base + j)) ? tx.w[e] : w;

		wx8[j] = vec ? w : 0.f;
	}

	for (int c = 0; c < C; c++) {

		float2 val = ksp[m + M * c];

		if ((0.f == val.x) && (0.f == val.y))
			continue;

		float2* gc = grid + g.gsz * c;
#pragma unroll 1
		for (int a = 0; a < TZ; a++) {

			float dz = tz.w[a];
			long oz = (long)tz.cell[a] * g.G[1];
#pragma unroll
			for (int b = 0; b < 6; b++) {

				float dzy = __fmul_rn(dz, ty.w[b]);
				long oy = (oz + ty.cell[b]) * g.G[0];

				if (0.f == dzy)
					continue;

				if (vec) {
#pragma unroll
					for (int q = 0; q < 4; q++) {

						float d0 = __fmul_rn(dzy, wx8[2 * q]);
						float d1 = __fmul_rn(dzy, wx8[2 * q + 1]);

						if ((0.f != d0) || (0.f != d1))
							atomicAdd((float4*)(gc + oy + base + 2 * q),
								make_float4(val.x * d0, val.y * d0, val.x * d1, val.y * d1));
					}

				} else {
#pragma unroll
					for (int e = 0; e < 6; e++) {

						float d = __fmul_rn(dzy, tx.w[e]);

						if (0.f != d)
							atomicAdd(&gc[oy + tx.cell[e]], make_float2(val.x * d, val.y * d));
					}
				}
			}
		}
	}
}

// Gridding, width 6, output-stationary (the default scatter) ------------------
//
// The grid is cut into tiles that are the sample bins (TX x LY x LZ cells of
// the centred oversampled grid). One warp job owns one tile and a group of
// coils: lane (line, grp) holds the TX x-cells of tile line (y, z) = line
// for CT coils in registers, so it accumulates without atomics. A sample's
// taps lie within 3 cells of its centred position 2k + N on every axis
// (cells 2w + s, |w - pos_s| <= 1.5), so the samples that reach a tile are
// in the tile's bin and its 3^d - 1 neighbours: the warp scans those bins'
// sorted samples 32 at a time, keeps the ones whose footprint meets the tile
// (ballot + compaction into shared memory, with their weights and coil
// values), and adds each kept sample to its lanes' cells. The x offset of a
// sample is the same for the whole warp, so a switch on it selects a fully
// unrolled update of exactly the taps inside the tile; lanes whose line is
// outside the sample's y/z window skip it.
//
// Work items: a tile's candidates (the samples of its neighbourhood, in a
// fixed bin order) are cut into chunks (TileWork.cand); tiles with one chunk
// write their cells with plain stores (empty tiles write zeros, so the grid
// needs no clearing), tiles with several chunks (the dense k-space centre)
// add their chunks with atomics into cells that k_zero_tiles cleared.
// Weights are those of axis_taps6 (bit-identical to the reference's
// grid_point_gen, src/noncart/grid.c:403-465) and the combined weight the
// same float32 product ((1 * wz) * wy) * wx.

enum { TG_WARPS = 4 };

struct TileWork {

	const int* bin_start;		// [nbins + 1] sorted sample range of each bin
	const int* work_tile;		// [nwork] tile of a work item
	const int* work_chunk;		// [nwork] chunk of the tile's candidates
	const int* nwork_dev;		// number of work items
	const unsigned char* multi;	// [ntiles] 1 if the tile has several work items
	const float4* foot;		// [M][FOOT_F4] footprints of the sorted samples
	int cand;			// candidates per work item
};

// Footprint record of a sorted sample (built once per trajectory by
// k_foot): float4 0 holds the centred start cells lo of the x, y, z taps
// (as int bits); float4s 1..5 the weights of cells lo .. lo + 5 per axis,
// x then y then z (6 each, the last two slots zero). A singleton axis has
// lo = 0 and the one weight intlookup(0).
enum { FOOT_F4 = 6 };

// Footprint of one axis: the six taps of a sample (two sub-grids x three)
// lie on the centred cells lo .. lo + 5 (2w + s); w7[t] is the weight of
// cell lo + t (0 where a non-periodic grid clips the tap). Singleton axis:
// one tap at 0 with weight intlookup(0).
__device__ __forceinline__ int foot6_lo(float k, int N)
{
	if (1 == N)
		return 0;

	const float half = (float)(N / 2);
	int lo = INT_MAX;
#pragma unroll
	for (int s = 0; s < 2; s++) {

		float pos = __fadd_rn(__fadd_rn(k, s ? -0.5f : -0.0f), half);
		double l = (double)pos - 1.5;
		int sti = (int)ceil(l);

		if ((double)sti == l)
			sti += 1;

		lo = min(lo, 2 * sti + s);
	}

	return lo;
}

__device__ __forceinline__ void foot6_w(float k, int N, int periodic, const float* kb, int lo, float* w7)
{
#pragma unroll
	for (int t = 0; t < 7; t++)
		w7[t] = 0.f;

	if (1 == N) {

		w7[0] = kb_lookup(kb, 0.f);
		return;
	}

	const float half = (float)(N / 2);
#pragma unroll
	for (int s = 0; s < 2; s++) {

		float pos = __fadd_rn(__fadd_rn(k, s ? -0.5f : -0.0f), half);
		double l = (double)pos - 1.5;
		int sti = (int)ceil(l);

		if ((double)sti == l)
			sti += 1;
#pragma unroll
		for (int q = 0; q < 3; q++) {

			int w = sti + q;
			float frac = fabsf(__fsub_rn((float)w, pos));
			float val = kb_lookup(kb, __fdiv_rn(frac, 3.0f));
			bool valid = periodic || ((w >= 0) && (w <= N - 1));
			int t = 2 * w + s - lo;

			if ((t >= 0) && (t < 7))
				w7[t] = valid ? val : 0.f;
		}
	}
}

// footprints of all sorted samples (the weights as axis_taps6 computes them:
// the same kb_lookup of the same float32 distances)
__global__ void k_foot(const float4* __restrict__ traj_sorted, long M, GridGeom g, const float* __restrict__ kbg,
		float4* __restrict__ foot)
{
	__shared__ float kb[KB_TABLE_N + 1];

	for (int i = threadIdx.x; i <= KB_TABLE_N; i += blockDim.x)
		kb[i] = kbg[i];

	__syncthreads();

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (long)gridDim.x * blockDim.x) {

		const float4 k = traj_sorted[i];
		const float kk[3] = { k.x, k.y, k.z };
		float w[24];
		int lo[3];
#pragma unroll
		for (int a = 0; a < 3; a++) {

			float w7[7];
			lo[a] = foot6_lo(kk[a], g.N[a]);
			foot6_w(kk[a], g.N[a], g.periodic, kb, lo[a], w7);
#pragma unroll
			for (int t = 0; t < 6; t++)
				w[6 * a + t] = w7[t];
		}

		w[18] = w[19] = w[20] = w[21] = w[22] = w[23] = 0.f;
		float4* f = foot + i * FOOT_F4;
		f[0] = make_float4(__int_as_float(lo[0]), __int_as_float(lo[1]), __int_as_float(lo[2]), 0.f);
#pragma unroll
		for (int q = 0; q < 5; q++)
			f[1 + q] = make_float4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
	}
}

// offset of a footprint start relative to a tile origin, along an axis of
// G cells: periodic grids take the representative nearest to the tile
__device__ __forceinline__ int foot_rel(int lo, int origin, int G, int periodic)
{
	int r = lo - origin;

	if (periodic) {

		r %= G;

		if (r > G / 2)
			r -= G;
		else if (r < -G / 2)
			r += G;
	}

	return r;
}

// DFT-order index of centred cell c of an axis (G = 2N cells; 0 for singletons)
__device__ __forceinline__ int dft_index(int c, int N, int G)
{
	if (1 == G)
		return 0;

	c += N;
	return (c >= G) ? c - G : c;
}

// one staged sample of a warp job
template <int CW>
struct __align__(16) TgSample {

	float w[24];		// x, y, z weights of cells lo .. lo + 5 (6 each)
	int rx, ry, rz, pad;
	float2 v[CW];
};

// acc[i][c] += (wyz * wx[t]) * v[c] for the taps t whose cell i = RX + t is
// inside the tile (RX a compile-time offset)
template <int TX, int CT, int RX>
__device__ __forceinline__ void tg_accum_x(float2 (&acc)[TX][CT], const float* wx, float wyz, const float2* v)
{
#pragma unroll
	for (int t = 0; t < 6; t++) {

		if ((RX + t >= 0) && (RX + t < TX)) {

			float d = __fmul_rn(wyz, wx[t]);
#pragma unroll
			for (int c = 0; c < CT; c++) {

				acc[RX + t][c].x = fmaf(v[c].x, d, acc[RX + t][c].x);
				acc[RX + t][c].y = fmaf(v[c].y, d, acc[RX + t][c].y);
			}
		}
	}
}

// the update for a sample at x offset rx (-5 .. TX - 1, at most 15)
#define BN_TG_CASE(R) case R: tg_accum_x<TX, CT, R>(acc, wx, wyz, v); break;

template <int TX, int CT>
__device__ __forceinline__ void tg_switch(int rx, float2 (&acc)[TX][CT], const float* wx, float wyz, const float2* v)
{
	static_assert(TX <= 16, "x offsets up to 15");

	switch (rx) {
	BN_TG_CASE(-5) BN_TG_CASE(-4) BN_TG_CASE(-3) BN_TG_CASE(-2) BN_TG_CASE(-1)
	BN_TG_CASE(0) BN_TG_CASE(1) BN_TG_CASE(2) BN_TG_CASE(3) BN_TG_CASE(4) BN_TG_CASE(5) BN_TG_CASE(6)
	BN_TG_CASE(7) BN_TG_CASE(8) BN_TG_CASE(9) BN_TG_CASE(10) BN_TG_CASE(11) BN_TG_CASE(12) BN_TG_CASE(13)
	BN_TG_CASE(14) BN_TG_CASE(15)
	default: break;
	}
}

#undef BN_TG_CASE

// grid cells of the tiles that several work items add into: zeroed first
__global__ void k_zero_tiles(float2* __restrict__ grid, GridGeom g, BinGeom bg, const unsigned char* __restrict__ multi,
		long ntiles, int C)
{
	const long per = (long)bg.bs[0] * bg.bs[1] * bg.bs[2];

	for (long t = blockIdx.x; t < ntiles; t += gridDim.x) {

		if (!multi[t])
			continue;

		const int bx = (int)(t % bg.nb[0]), by = (int)((t / bg.nb[0]) % bg.nb[1]), bz = (int)(t / ((long)bg.nb[0] * bg.nb[1]));

		for (long e = threadIdx.x; e < per * C; e += blockDim.x) {

			const int c = (int)(e / per);
			const long l = e - (long)c * per;
			const int cx = bx * bg.bs[0] + (int)(l % bg.bs[0]);
			const int cy = by * bg.bs[1] + (int)((l / bg.bs[0]) % bg.bs[1]);
			const int cz = bz * bg.bs[2] + (int)(l / ((long)bg.bs[0] * bg.bs[1]));

			if ((cx >= g.G[0]) || (cy >= g.G[1]) || (cz >= g.G[2]))
				continue;

			const long cell = dft_index(cx, g.N[0], g.G[0]) + (long)g.G[0] * (dft_index(cy, g.N[1], g.G[1])
					+ (long)g.G[1] * dft_index(cz, g.N[2], g.G[2]));
			grid[cell + g.gsz * c] = make_float2(0.f, 0.f);
		}
	}
}

// candidates of tile (tx, ty, tz): the neighbour bins in the order dz, dy,
// dx = -1..1 (singleton axes: 0 only; non-periodic edges skipped)
__device__ __forceinline__ int tg_neighbour(int b, int d, int nb, int periodic)
{
	int n = b + d;

	if (periodic)
		return (n < 0) ? n + nb : ((n >= nb) ? n - nb : n);

	return ((n < 0) || (n >= nb)) ? -1 : n;
}

// candidates per tile and the work items (chunks of cand) per tile
__global__ void k_tile_cand(const int* __restrict__ bin_start, BinGeom bg, int periodic, long ntiles, int cand,
		int* __restrict__ nwork, unsigned char* __restrict__ multi)
{
	for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += (long)gridDim.x * blockDim.x) {

		const int bx = (int)(t % bg.nb[0]), by = (int)((t / bg.nb[0]) % bg.nb[1]), bz = (int)(t / ((long)bg.nb[0] * bg.nb[1]));
		const int rz = (bg.nb[2] > 1) ? 1 : 0, ry = (bg.nb[1] > 1) ? 1 : 0;
		long n = 0;

		for (int dz = -rz; dz <= rz; dz++) {

			const int z = tg_neighbour(bz, dz, bg.nb[2], periodic);

			if (z < 0)
				continue;

			for (int dy = -ry; dy <= ry; dy++) {

				const int y = tg_neighbour(by, dy, bg.nb[1], periodic);

				if (y < 0)
					continue;

				for (int dx = -1; dx <= 1; dx++) {

					const int x = tg_neighbour(bx, dx, bg.nb[0], periodic);

					if (x < 0)
						continue;

					const long b = x + (long)bg.nb[0] * (y + (long)bg.nb[1] * z);
					n += bin_start[b + 1] - bin_start[b];
				}
			}
		}

		const long w = (n + cand - 1) / cand;
		nwork[t] = (int)((w < 1) ? 1 : w);
		multi[t] = (w > 1) ? 1 : 0;
	}
}

// work item table: tile t owns items work_start[t] .. work_start[t + 1] - 1
__global__ void k_work_fill(const int* __restrict__ work_start, long ntiles, int* __restrict__ work_tile,
		int* __restrict__ work_chunk)
{
	for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += (long)gridDim.x * blockDim.x)
		for (int w = work_start[t]; w < work_start[t + 1]; w++) {

			work_tile[w] = (int)t;
			work_chunk[w] = w - work_start[t];
		}
}

// TX x-cells per lane, LY x LZ lines per tile (LY * LZ divides 32), CT coils
// per lane: a warp job covers CW = (32 / (LY * LZ)) * CT coils. ksp_sorted:
// ksp is in bin order (sample i of the sorted trajectory at ksp[i + M c]),
// else in the caller's order (ksp[perm[i] + M c]).
template <int TX, int LY, int LZ, int CT>
__global__ void __launch_bounds__(32 * TG_WARPS, 4) k_grid6_tiles(const int* __restrict__ perm, long M, GridGeom g,
		BinGeom bg, TileWork tw, int C, const float2* __restrict__ ksp, int ksp_sorted, float2* __restrict__ grid)
{
	constexpr int NL = LY * LZ;
	constexpr int GPW = 32 / NL;
	constexpr int CW = GPW * CT;
	static_assert(NL * GPW == 32, "lines per tile must divide 32");
	__shared__ TgSample<CW> stage[TG_WARPS][32];

	const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
	const int ncq = (C + CW - 1) / CW;	// coil chunks
	const long job = (long)blockIdx.x * TG_WARPS + warp;
	const long wi = job / ncq;
	const int cq = (int)(job % ncq);

	if (wi >= *tw.nwork_dev)	// warp-uniform; the warps share no barrier
		return;

	const int tile = tw.work_tile[wi];
	const int chunk = tw.work_chunk[wi];
	const int bx = tile % bg.nb[0], by = (tile / bg.nb[0]) % bg.nb[1], bz = tile / (bg.nb[0] * bg.nb[1]);
	const int ox = bx * TX, oy = by * LY, oz = bz * LZ;
	const int j = lane % LY, k = (lane / LY) % LZ, grp = lane / NL;
	const int cw0 = cq * CW;		// first coil of the job
	const int c0 = cw0 + grp * CT;		// first coil of this lane
	TgSample<CW>* sg = stage[warp];

	float2 acc[TX][CT];
#pragma unroll
	for (int i = 0; i < TX; i++)
#pragma unroll
		for (int c = 0; c < CT; c++)
			acc[i][c] = make_float2(0.f, 0.f);

	const long cand0 = (long)chunk * tw.cand, cand1 = cand0 + tw.cand;
	const int rz = (bg.nb[2] > 1) ? 1 : 0, ry = (bg.nb[1] > 1) ? 1 : 0;
	long off = 0;

	for (int dz = -rz; (dz <= rz) && (off < cand1); dz++) {

		const int nz = tg_neighbour(bz, dz, bg.nb[2], g.periodic);

		if (nz < 0)
			continue;

		for (int dy = -ry; (dy <= ry) && (off < cand1); dy++) {

			const int ny = tg_neighbour(by, dy, bg.nb[1], g.periodic);

			if (ny < 0)
				continue;

			for (int dx = -1; (dx <= 1) && (off < cand1); dx++) {

				const int nx = tg_neighbour(bx, dx, bg.nb[0], g.periodic);

				if (nx < 0)
					continue;

				const long b = nx + (long)bg.nb[0] * (ny + (long)bg.nb[1] * nz);
				const int s0 = tw.bin_start[b], s1 = tw.bin_start[b + 1];
				const long a = max(off, cand0), e = min(off + (long)(s1 - s0), cand1);
				const int i0 = s0 + (int)(a - off), i1 = s0 + (int)(e - off);
				off += s1 - s0;

				// batches of 32 candidates; the next batch's footprint start
				// and coil values are loaded while this batch accumulates
				float4 f0n = make_float4(0.f, 0.f, 0.f, 0.f);
				float2 vn[CW];

				auto fetch = [&](int i) {
					if (i < i1) {

						f0n = tw.foot[(long)i * FOOT_F4];
						const long m = ksp_sorted ? (long)i : (long)perm[i];
#pragma unroll
						for (int c = 0; c < CW; c++)
							vn[c] = (cw0 + c < C) ? ksp[m + M * (cw0 + c)] : make_float2(0.f, 0.f);
					}
				};

				fetch(i0 + lane);

				for (int base = i0; base < i1; base += 32) {

					const int i = base + lane;
					const float4 f0 = f0n;
					float2 vc[CW];
#pragma unroll
					for (int c = 0; c < CW; c++)
						vc[c] = vn[c];

					fetch(i + 32);
					bool hit = false;
					int lx = 0, ly = 0, lz = 0;

					if (i < i1) {

						lx = foot_rel(__float_as_int(f0.x), ox, g.G[0], g.periodic);
						ly = foot_rel(__float_as_int(f0.y), oy, g.G[1], g.periodic);
						lz = foot_rel(__float_as_int(f0.z), oz, g.G[2], g.periodic);
						hit = (lx > -6) && (lx < TX) && (ly > -6) && (ly < LY) && (lz > -6) && (lz < LZ);
					}

					const unsigned mask = __ballot_sync(0xffffffffu, hit);
					const int n = __popc(mask);

					if (hit) {

						TgSample<CW>& d = sg[__popc(mask & ((1u << lane) - 1u))];
						const float4* f = tw.foot + (long)i * FOOT_F4;
#pragma unroll
						for (int q = 0; q < 5; q++)
							*(float4*)(d.w + 4 * q) = f[1 + q];
						d.rx = lx;
						d.ry = ly;
						d.rz = lz;
#pragma unroll
						for (int c = 0; c < CW; c++)
							d.v[c] = vc[c];
					}

					__syncwarp();

					for (int q = 0; q < n; q++) {

						const TgSample<CW>& d = sg[q];
						const int ty = j - d.ry, tz = k - d.rz;

						if ((ty < 0) || (ty >= 6) || (tz < 0) || (tz >= 6))
							continue;

						const float wyz = __fmul_rn(d.w[12 + tz], d.w[6 + ty]);

						if (0.f == wyz)
							continue;

						float2 v[CT];
#pragma unroll
						for (int c = 0; c < CT; c++)
							v[c] = d.v[grp * CT + c];

						tg_switch<TX, CT>(d.rx, acc, d.w, wyz, v);
					}

					__syncwarp();
				}
			}
		}
	}

	// this lane's line: TX cells from ox along x, at (oy + j, oz + k)
	const int cy = oy + j, cz = oz + k;

	if ((cy >= g.G[1]) || (cz >= g.G[2]))
		return;

	const bool add = tw.multi[tile];
	const long row = (long)g.G[0] * (dft_index(cy, g.N[1], g.G[1]) + (long)g.G[1] * dft_index(cz, g.N[2], g.G[2]));
#pragma unroll
	for (int i = 0; i < TX; i++) {

		const int cx = ox + i;

		if (cx >= g.G[0])
			break;

		const long cell = row + dft_index(cx, g.N[0], g.G[0]);
#pragma unroll
		for (int c = 0; c < CT; c++) {

			if (c0 + c >= C)
				break;

			float2* dst = grid + cell + g.gsz * (c0 + c);

			if (add)
				atomicAdd(dst, acc[i][c]);
			else
				*dst = acc[i][c];
		}
	}
}

// ksp [M, C] into bin order: dst[i + M c] = src[perm[i] + M c]
__global__ void k_permute_ksp(float2* __restrict__ dst, const float2* __restrict__ src, const int* __restrict__ perm,
		long M, int C)
{
	for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < M * C; e += (long)gridDim.x * blockDim.x) {

		const long c = e / M, i = e - c * M;
		dst[e] = src[perm[i] + M * c];
	}
}

} // namespace bn
