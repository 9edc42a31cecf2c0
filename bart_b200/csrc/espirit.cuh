// ESPIRiT calibration (bart ecalib) on the GPU: the reference's default
// path (src/ecalib.c:46-262, src/calib/calib.c) as
//
//   calibration region (host search over the centre block's coil energies)
//   -> Casorati matrix of the region's kernel-sized patches
//   -> Gram matrix (tiled complex GEMM)
//   -> Hermitian eigen-decomposition (cuSOLVER cheevd, the one library
//      call: the reference calls LAPACK cheev here)
//   -> kernel images on the (2k)^d grid (DFT as a complex GEMM) and their
//      packed C x C Gram matrix per low-resolution pixel
//   -> sinc interpolation along y and z to every image row
//   -> one fused pass per image pixel: sinc interpolation along x, the
//      orthogonal iteration, eigenvalue crop and phase alignment, written
//      straight to the maps [X, Y, Z, C, maps].
// The covariance is accumulated and interpolated in float64 (it is small
// and the result of cancellation away from the object); the GEMMs, the
// eigen-decomposition and the orthogonal iteration run in float32, as the
// reference's do.
//
// This file is included into bnufft.cu and uses its error and launch
// helpers (fail, CUDA_TRY, LAUNCHED, TRY, on_device).

#include <dlfcn.h>
#include <cusolverDn.h>

#include <algorithm>
#include <thread>
#include <type_traits>

#include "../../include/bespirit.h"

namespace bn {

// ---------------------------------------------------------------------------
// device kernels
// ---------------------------------------------------------------------------

__device__ __forceinline__ float2 ec_cmulc(float2 a, float2 b) { return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }	// a conj(b)
__device__ __forceinline__ float2 ec_conj(float2 a) { return make_float2(a.x, -a.y); }

// dst[bx, by, bz, C] (contiguous) = src[ox + x, oy + y, oz + z, c] of a
// [X, Y, Z, C] array.
__global__ void k_ec_gather(const float2* __restrict__ src, long X, long Y, long Z, int C, int ox, int oy, int oz,
			    int bx, int by, int bz, float2* __restrict__ dst)
{
	const long n = (long)bx * by * bz * C;

	for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		long t = i;
		const int x = (int)(t % bx); t /= bx;
		const int y = (int)(t % by); t /= by;
		const int z = (int)(t % bz);
		const int c = (int)(t / bz);
		dst[i] = src[(ox + x) + X * ((oy + y) + Y * ((oz + z) + Z * (long)c))];
	}
}

// Coil energy of every voxel of the centre block [bx, by, bz] of a
// [X, Y, Z, C] array at (ox, oy, oz): e = sum_c |v|^2 (double sums rounded
// once). Zero exactly where the reference's pattern (root-sum-of-squares
// != 0, src/misc/mri2.c:39-57) is zero.
__global__ void k_ec_energy(const float2* __restrict__ src, long X, long Y, long Z, int C, int ox, int oy, int oz,
			    int bx, int by, int bz, float* __restrict__ e)
{
	const long n = (long)bx * by * bz;

	for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		const int x = (int)(i % bx), y = (int)((i / bx) % by), z = (int)(i / ((long)bx * by));
		const float2* p = src + (ox + x) + X * ((oy + y) + Y * (long)(oz + z));
		double s = 0.;

		for (int c = 0; c < C; c++) {

			const float2 v = p[X * Y * Z * (long)c];
			s += (double)v.x * v.x + (double)v.y * v.y;
		}

		e[i] = (float)s;
	}
}

// Casorati matrix A [P][Ncol] (row-major): A[p][j] = cal[p + k_j, c_j] with
// j = kx_i + kx (ky_i + ky (kz_i + kz c)) (src/num/casorati.c:34-65).
__global__ void k_ec_casorati(const float2* __restrict__ cal, int cx, int cy, int cz, int kx, int ky, int kz, int C,
			      float2* __restrict__ A)
{
	const int px = cx - kx + 1, py = cy - ky + 1, pz = cz - kz + 1;
	const long P = (long)px * py * pz;
	const long ncol = (long)kx * ky * kz * C;

	for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < P * ncol; i += (long)gridDim.x * blockDim.x) {

		const long p = i / ncol;
		long j = i % ncol;
		const int jx = (int)(j % kx); j /= kx;
		const int jy = (int)(j % ky); j /= ky;
		const int jz = (int)(j % kz);
		const int c = (int)(j / kz);
		const int x = (int)(p % px), y = (int)((p / px) % py), z = (int)(p / ((long)px * py));
		A[i] = cal[(x + jx) + (long)cx * ((y + jy) + (long)cy * ((z + jz) + (long)cz * c))];
	}
}

// C [M][N] = op(A) [M][K] * op(B) [K][N], row-major complex float, 64 x 64
// tiles, 4 x 4 outputs per thread. CONJ_A: op(A) = A^H with A stored
// [K][M]; else A stored [M][K]. CONJ_BT: op(B) = B^H with B stored [N][K];
// else B stored [K][N].
// LOWER: only the tiles that hold entries with row >= column are computed
// (a Hermitian Gram matrix for the eigen-decomposition, which reads the
// row-major lower triangle: UPLO 'U' of its column-major view); the tiles
// above are written as zeros.
template <bool CONJ_A, bool CONJ_BT, bool LOWER = false>
__global__ void __launch_bounds__(256) k_ec_cgemm(int M, int N, int K, const float2* __restrict__ A, long lda,
						  const float2* __restrict__ B, long ldb, float2* __restrict__ Cm, long ldc)
{
	__shared__ float2 As[16][64 + 1];
	__shared__ float2 Bs[16][64 + 1];

	const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
	const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;

	if (LOWER && n0 > m0 + 63) {

		for (int i = 0; i < 4; i++)
			for (int j = 0; j < 4; j++) {

				const int gm = m0 + ty * 4 + i, gn = n0 + tx * 4 + j;

				if (gm < M && gn < N)
					Cm[gm * ldc + gn] = make_float2(0.f, 0.f);
			}

		return;
	}

	float2 acc[4][4];

	for (int i = 0; i < 4; i++)
		for (int j = 0; j < 4; j++)
			acc[i][j] = make_float2(0.f, 0.f);

	for (int k0 = 0; k0 < K; k0 += 16) {

		for (int e = threadIdx.x; e < 1024; e += 256) {

			int kk, mm;

			if (CONJ_A) {

				kk = e / 64;
				mm = e % 64;

			} else {

				mm = e / 16;
				kk = e % 16;
			}

			const int gm = m0 + mm, gk = k0 + kk;
			float2 a = make_float2(0.f, 0.f);

			if (gm < M && gk < K)
				a = CONJ_A ? ec_conj(A[gk * lda + gm]) : A[gm * lda + gk];

			As[kk][mm] = a;

			const int nn = CONJ_BT ? e / 16 : e % 64, kb = CONJ_BT ? e % 16 : e / 64;
			const int gn = n0 + nn, gkb = k0 + kb;
			float2 b = make_float2(0.f, 0.f);

			if (gn < N && gkb < K)
				b = CONJ_BT ? ec_conj(B[gn * ldb + gkb]) : B[gkb * ldb + gn];

			Bs[kb][nn] = b;
		}

		__syncthreads();

#pragma unroll
		for (int kk = 0; kk < 16; kk++) {

			float2 a[4], b[4];

			for (int i = 0; i < 4; i++)
				a[i] = As[kk][ty * 4 + i];

			for (int j = 0; j < 4; j++)
				b[j] = Bs[kk][tx * 4 + j];

			for (int i = 0; i < 4; i++)
				for (int j = 0; j < 4; j++) {

					acc[i][j].x = fmaf(a[i].x, b[j].x, fmaf(-a[i].y, b[j].y, acc[i][j].x));
					acc[i][j].y = fmaf(a[i].x, b[j].y, fmaf(a[i].y, b[j].x, acc[i][j].y));
				}
		}

		__syncthreads();
	}

	for (int i = 0; i < 4; i++)
		for (int j = 0; j < 4; j++) {

			const int gm = m0 + ty * 4 + i, gn = n0 + tx * 4 + j;

			if (gm < M && gn < N)
				Cm[gm * ldc + gn] = acc[i][j];
		}
}

// Kernels in descending eigenvalue order, arranged for the kernel-image
// GEMM: KT[u][c n + i] = E[N - 1 - i][u + kd c] (E row-major: row r is the
// eigenvector of the r-th smallest eigenvalue, as LAPACK returns them).
__global__ void k_ec_kern_perm(const float2* __restrict__ E, int Ncol, int kd, int C, int n, float2* __restrict__ KT)
{
	const long tot = (long)kd * C * n;

	for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {

		const int u = (int)(t / ((long)C * n));
		const int r = (int)(t % ((long)C * n));
		const int c = r / n, i = r % n;
		KT[t] = E[(long)(Ncol - 1 - i) * Ncol + u + (long)kd * c];
	}
}

// The same arrangement when the eigenvectors u_i are those of the P x P
// matrix A A^H (fewer patches than kernel entries): kernel i is
// A^T u_(P-1-i) / sigma_i, the right singular vector of conj(A), i.e. the
// eigenvector of conj(G) that LAPACK returns in the reference.
__global__ void k_ec_kern_left(const float2* __restrict__ A, const float2* __restrict__ E, int P, int Ncol, int kd, int C,
			       int n, const float* __restrict__ inv_sigma, float2* __restrict__ KT)
{
	const long tot = (long)kd * C * n;

	for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {

		const int u = (int)(t / ((long)C * n));
		const int r = (int)(t % ((long)C * n));
		const int c = r / n, i = r % n;
		const long j = u + (long)kd * c;
		const float2* e = E + (long)(P - 1 - i) * P;
		double sr = 0., si = 0.;

		for (int p = 0; p < P; p++) {

			const float2 a = A[(long)p * Ncol + j], w = e[p];
			sr += (double)a.x * w.x - (double)a.y * w.y;
			si += (double)a.x * w.y + (double)a.y * w.x;
		}

		KT[t] = make_float2((float)(sr * inv_sigma[i]), (float)(si * inv_sigma[i]));
	}
}

// Packed lower-triangular Gram matrix of the kernel images per
// low-resolution pixel: cov[x][l(a, b)] = sum_i conj(K[x][a n + i])
// K[x][b n + i] * scale, l(a, b) = a (a + 1) / 2 + b, b <= a
// (src/calib/calib.c:1072-1088, src/num/linalg.c:642-664, 1211-1232).
__global__ void k_ec_pixgram(const float2* __restrict__ Kimg, int C, int n, double scale, double2* __restrict__ cov)
{
	const int x = blockIdx.x;
	const int L = C * (C + 1) / 2;
	const float2* K = Kimg + (long)x * C * n;

	for (int l = threadIdx.x; l < L; l += blockDim.x) {

		int a = (int)((sqrtf(8.f * l + 1.f) - 1.f) * 0.5f);

		while (a * (a + 1) / 2 > l)
			a--;

		while ((a + 1) * (a + 2) / 2 <= l)
			a++;

		const int b = l - a * (a + 1) / 2;
		const float2* ka = K + (long)a * n;
		const float2* kb = K + (long)b * n;
		double sr = 0., si = 0.;

		for (int i = 0; i < n; i++) {

			const float2 p = ka[i], q = kb[i];	// conj(p) q
			sr = fma((double)p.x, (double)q.x, fma((double)p.y, (double)q.y, sr));
			si = fma((double)p.x, (double)q.y, fma(-(double)p.y, (double)q.x, si));
		}

		cov[(long)x * L + l] = make_double2(sr * scale, si * scale);
	}
}

// [hd][L] float64 -> [L][hd] float32 (calone's output layout)
__global__ void k_ec_cov_layout(const double2* __restrict__ cov, long hd, long L, float2* __restrict__ out)
{
	for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < hd * L; t += (long)gridDim.x * blockDim.x) {

		const long x = t % hd, l = t / hd;
		const double2 v = cov[x * L + l];
		out[t] = make_float2((float)v.x, (float)v.y);
	}
}

// sinc interpolation along y and z (the reference's sinc_zeropad,
// src/misc/resize.c:234-292, written as its per-axis linear maps):
// T[(z Y + y)][u][l] = sum_{v, w} Ry[y][v] Rz[z][w] cov[(w yh + v) xh + u][l].
// In float64: away from the object the interpolated covariance is a small
// difference of order-one terms, and its relative error there sets the
// accuracy of the maps wherever the eigenvalues lie close together.
__global__ void k_ec_interp_yz(const double2* __restrict__ cov, int xh, int yh, int zh, int L, int Y,
			       const double2* __restrict__ Ry, const double2* __restrict__ Rz, double2* __restrict__ T)
{
	const int row = blockIdx.x;
	const int y = row % Y, z = row / Y;
	const int n = xh * L;

	for (int t = threadIdx.x; t < n; t += blockDim.x) {

		const int u = t / L, l = t % L;
		double2 s = make_double2(0., 0.);

		for (int w = 0; w < zh; w++) {

			const double2 rz = Rz[(long)z * zh + w];

			for (int v = 0; v < yh; v++) {

				const double2 ry = Ry[(long)y * yh + v];
				const double2 r = make_double2(ry.x * rz.x - ry.y * rz.y, ry.x * rz.y + ry.y * rz.x);
				const double2 c = cov[((long)(w * yh + v) * xh + u) * L + l];
				s.x = fma(r.x, c.x, fma(-r.y, c.y, s.x));
				s.y = fma(r.x, c.y, fma(r.y, c.x, s.y));
			}
		}

		T[(long)row * n + t] = s;
	}
}

template <int W>
__device__ __forceinline__ float ec_group_sum(float v)
{
#pragma unroll
	for (int o = W / 2; o > 0; o >>= 1)
		v += __shfl_xor_sync(0xffffffffu, v, o);

	return v;
}

// One pass per image pixel: W lanes per pixel (lane c = coil c, W >= C,
// 32 / W pixels per warp), PX = 8 * 32 / W consecutive pixels of one image
// row per block.
//   1. lane c builds column c of the pixel's C x C Hermitian matrix from
//      the row's y/z-interpolated packed covariance (shared memory) and
//      the x-interpolation row Rx[x] (the upper triangle is the conjugate
//      of the lower, src/calib/calib.c:73-86);
//   2. iters steps of orthogonal iteration: rows v_m <- v_m H (the
//      coefficients broadcast through shared memory), then Gram-Schmidt
//      from the last row to the first (src/num/linalg.c:1235-1313); the
//      last row is the principal eigenvector;
//   3. map u = row M-1-u with eigenvalue = that row's last norm
//      (src/calib/calib.c:474-483); with intensity correction scaled to
//      l1 norm sqrt(C) over the coils; weight 0/1 for |e| >= crop, or the
//      reference's soft s-curve (src/calib/calib.c:88-134);
//   4. phase: times conj of the phase of sum_c map[c] conj(rot[c])
//      (src/misc/utils.c:148-174);
//   5. staged through shared memory and written coalesced along x.
template <int W, int MMAX>
__global__ void __launch_bounds__(256) k_ec_eigen(int X, int Y, int Z, int C, int M, int xh, int L,
						  const double2* __restrict__ T, const double2* __restrict__ Rx,
						  const float2* __restrict__ rot, int iters, float crop, int soft, int intensity,
						  float2* __restrict__ sens, float2* __restrict__ ev)
{
	constexpr int PX = 8 * 32 / W;
	constexpr int G = 32 / W;			// pixels per warp
	extern __shared__ double2 ec_smem[];
	double2* sT = ec_smem;				// [xh][L]
	double2* sR = sT + (long)xh * L;		// [PX][xh]
	float2* sV = (float2*)(sR + PX * xh);		// [warp][k][g][MMAX]: the iterates, for broadcast
	float2* sO = sV + 8 * W * G * MMAX;		// [PX][M][C]
	float* sE = (float*)(sO + PX * M * C);		// [PX][M]

	const int row = blockIdx.x;
	const int y = row % Y, z = row / Y;
	const int x0 = blockIdx.y * PX;
	const double2* Trow = T + (long)row * xh * L;

	for (int t = threadIdx.x; t < xh * L; t += blockDim.x)
		sT[t] = Trow[t];

	for (int t = threadIdx.x; t < PX * xh; t += blockDim.x) {

		const int px = t / xh, u = t % xh;
		sR[t] = (x0 + px < X) ? Rx[(long)(x0 + px) * xh + u] : make_double2(0., 0.);
	}

	__syncthreads();

	const int lane = threadIdx.x % 32;
	const int c = lane % W;
	const int g = lane / W;
	const int px = (threadIdx.x / 32) * G + g;
	float2* vw = sV + (threadIdx.x / 32) * (W * G * MMAX);
	const bool act = c < C;
	const double2* rx = sR + px * xh;

	float2 Hc[W];

#pragma unroll
	for (int k = 0; k < W; k++) {

		double2 s = make_double2(0., 0.);

		if (act && k < C) {

			const bool lo = c <= k;
			const int l = lo ? k * (k + 1) / 2 + c : c * (c + 1) / 2 + k;

			for (int u = 0; u < xh; u++) {

				const double2 r = rx[u], v = sT[u * L + l];
				s.x = fma(r.x, v.x, fma(-r.y, v.y, s.x));
				s.y = fma(r.x, v.y, fma(r.y, v.x, s.y));
			}

			if (!lo)
				s.y = -s.y;
		}

		Hc[k] = make_float2((float)s.x, (float)s.y);
	}

	float2 v[MMAX];
	float val[MMAX];

#pragma unroll
	for (int m = 0; m < MMAX; m++) {

		v[m] = make_float2((m < M && c == m) ? 1.f : 0.f, 0.f);
		val[m] = 0.f;
	}

	for (int it = 0; it < iters; it++) {

		// rows v_m <- v_m H. With 16 or 32 lanes per pixel the coefficients
		// v_m[k] reach every lane through shared memory, two rows per
		// 16-byte load; with 8 (four pixels per warp) by shuffles, which
		// measured faster there.
		if (W >= 16) {

#pragma unroll
			for (int m = 0; m < MMAX; m++)
				vw[(c * G + g) * MMAX + m] = v[m];

			__syncwarp();

#pragma unroll
			for (int p = 0; p < MMAX / 2; p++) {

				if (2 * p >= M)
					continue;

				float4 e = make_float4(0.f, 0.f, 0.f, 0.f);	// (row 2p, row 2p+1)

#pragma unroll
				for (int k = 0; k < W; k++) {

					const float4 a = *(const float4*)&vw[(k * G + g) * MMAX + 2 * p];
					e.x = fmaf(a.x, Hc[k].x, fmaf(-a.y, Hc[k].y, e.x));
					e.y = fmaf(a.x, Hc[k].y, fmaf(a.y, Hc[k].x, e.y));
					e.z = fmaf(a.z, Hc[k].x, fmaf(-a.w, Hc[k].y, e.z));
					e.w = fmaf(a.z, Hc[k].y, fmaf(a.w, Hc[k].x, e.w));
				}

				v[2 * p] = make_float2(e.x, e.y);
				v[2 * p + 1] = make_float2(e.z, e.w);
			}

			__syncwarp();

		} else {

#pragma unroll
			for (int m = 0; m < MMAX; m++) {

				if (m >= M)
					continue;

				float2 t = make_float2(0.f, 0.f);

#pragma unroll
				for (int k = 0; k < W; k++) {

					const float2 a = make_float2(__shfl_sync(0xffffffffu, v[m].x, k, W), __shfl_sync(0xffffffffu, v[m].y, k, W));
					t.x = fmaf(a.x, Hc[k].x, fmaf(-a.y, Hc[k].y, t.x));
					t.y = fmaf(a.x, Hc[k].y, fmaf(a.y, Hc[k].x, t.y));
				}

				v[m] = t;
			}
		}

#pragma unroll
		for (int m = MMAX - 1; m >= 0; m--) {

			if (m >= M)
				continue;

#pragma unroll
			for (int j = m + 1; j < MMAX; j++) {

				if (j >= M)
					continue;

				const float2 p = ec_cmulc(v[m], v[j]);
				const float sr = ec_group_sum<W>(p.x), si = ec_group_sum<W>(p.y);
				v[m].x -= sr * v[j].x - si * v[j].y;
				v[m].y -= sr * v[j].y + si * v[j].x;
			}

			const float nrm = sqrtf(ec_group_sum<W>(v[m].x * v[m].x + v[m].y * v[m].y));
			val[m] = nrm;
			const float inv = (nrm > 0.f) ? 1.f / nrm : 0.f;
			v[m].x *= inv;
			v[m].y *= inv;
		}
	}

#pragma unroll
	for (int u = 0; u < MMAX; u++) {

		if (u >= M)
			continue;

		const int r = M - 1 - u;
		float2 mv = make_float2(0.f, 0.f);
		float e = 0.f;

#pragma unroll
		for (int q = 0; q < MMAX; q++)
			if (q == r) {

				mv = v[q];
				e = val[q];
			}

		if (intensity) {	// l1 norm over the coils to sqrt(C), src/misc/utils.c:83-109

			const float l1 = ec_group_sum<W>(sqrtf(mv.x * mv.x + mv.y * mv.y));
			const float f = (0.f == l1) ? 0.f : sqrtf((float)C) / l1;
			mv.x *= f;
			mv.y *= f;
		}

		float w;

		if (soft) {

			const float t = (sqrtf(fabsf(e)) - crop) / (1.f - crop);
			w = ((t >= 1.f) ? 1.f : 0.f) + ((t >= -1.f) ? (t / (t * t + 1.f) + 0.5f) : 0.f);

		} else {

			w = (fabsf(e) >= crop) ? 1.f : 0.f;
		}

		mv.x *= w;
		mv.y *= w;

		const float2 rc = act ? rot[c] : make_float2(0.f, 0.f);
		const float2 p = ec_cmulc(mv, rc);
		const float sr = ec_group_sum<W>(p.x), si = ec_group_sum<W>(p.y);
		const float a = sqrtf(sr * sr + si * si);
		const float2 ph = (a == 0.f) ? make_float2(1.f, 0.f) : make_float2(sr / a, si / a);
		const float2 o = ec_cmulc(mv, ph);

		if (act)
			sO[(px * M + u) * C + c] = o;

		if (0 == c)
			sE[px * M + u] = e;
	}

	__syncthreads();

	const long npix = (long)X * Y * Z;
	const long base = (long)x0 + (long)X * (y + (long)Y * z);
	const int nx = min(PX, X - x0);

	for (int t = threadIdx.x; t < PX * M * C; t += blockDim.x) {

		const int p = t % PX, cu = t / PX;
		const int cc = cu % C, u = cu / C;

		if (p < nx)
			sens[base + p + npix * (cc + (long)C * u)] = sO[(p * M + u) * C + cc];
	}

	if (nullptr != ev)
		for (int t = threadIdx.x; t < PX * M; t += blockDim.x) {

			const int p = t % PX, u = t / PX;

			if (p < nx)
				ev[base + p + npix * u] = make_float2(sE[p * M + u], 0.f);
		}
}

// coil covariance of the calibration data, row-major [C][C]:
// Gc[i][j] = sum_p conj(d_i[p]) d_j[p] (src/calib/cc.c:56-57,
// src/num/linalg.c:642-654)
__global__ void k_ec_coilcov(const float2* __restrict__ cal, long csize, int C, float2* __restrict__ Gc)
{
	const int i = blockIdx.x / C, j = blockIdx.x % C;
	const float2* a = cal + csize * i;
	const float2* b = cal + csize * j;
	double sr = 0., si = 0.;

	for (long p = threadIdx.x; p < csize; p += blockDim.x) {

		const float2 x = a[p], y = b[p];
		sr += (double)x.x * y.x + (double)x.y * y.y;
		si += (double)x.x * y.y - (double)x.y * y.x;
	}

	__shared__ double rr[256], ri[256];
	rr[threadIdx.x] = sr;
	ri[threadIdx.x] = si;
	__syncthreads();

	for (int o = blockDim.x / 2; o > 0; o >>= 1) {

		if ((int)threadIdx.x < o) {

			rr[threadIdx.x] += rr[threadIdx.x + o];
			ri[threadIdx.x] += ri[threadIdx.x + o];
		}

		__syncthreads();
	}

	if (0 == threadIdx.x)
		Gc[blockIdx.x] = make_float2((float)rr[0], (float)ri[0]);
}

}	// namespace bn

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

// cuSOLVER, loaded on first use so that the NUFFT / CG entry points keep
// depending on the CUDA runtime alone.
struct EcSolver {

	cusolverStatus_t (*create)(cusolverDnHandle_t*);
	cusolverStatus_t (*destroy)(cusolverDnHandle_t);
	cusolverStatus_t (*set_stream)(cusolverDnHandle_t, cudaStream_t);
	cusolverStatus_t (*heevd_size)(cusolverDnHandle_t, cusolverEigMode_t, cublasFillMode_t, int, const cuComplex*, int, const float*, int*);
	cusolverStatus_t (*heevd)(cusolverDnHandle_t, cusolverEigMode_t, cublasFillMode_t, int, cuComplex*, int, float*, cuComplex*, int, int*);
};

static int ec_solver(const EcSolver** out)
{
	static EcSolver api;
	static int state = 0;	// 0 unloaded, 1 ok, 2 failed
	static std::mutex mu;
	std::lock_guard<std::mutex> lock(mu);

	if (0 == state) {

		void* h = dlopen("libcusolver.so.11", RTLD_NOW | RTLD_LOCAL);

		if (nullptr == h)
			h = dlopen("libcusolver.so", RTLD_NOW | RTLD_LOCAL);

		state = 2;

		if (nullptr != h) {

			api.create = (decltype(api.create))dlsym(h, "cusolverDnCreate");
			api.destroy = (decltype(api.destroy))dlsym(h, "cusolverDnDestroy");
			api.set_stream = (decltype(api.set_stream))dlsym(h, "cusolverDnSetStream");
			api.heevd_size = (decltype(api.heevd_size))dlsym(h, "cusolverDnCheevd_bufferSize");
			api.heevd = (decltype(api.heevd))dlsym(h, "cusolverDnCheevd");

			if (api.create && api.destroy && api.set_stream && api.heevd_size && api.heevd)
				state = 1;
		}
	}

	if (1 != state)
		return fail(BNUFFT_ERR_CUDA, "ecalib: cuSOLVER (libcusolver.so.11) not available");

	*out = &api;
	return BNUFFT_OK;
}

// the calibration's own stream-ordered memory pool per device: no
// device-wide synchronisation per allocation, and (release threshold
// unlimited) the memory stays mapped for the next calibration instead of
// going back to the system at every synchronisation
static cudaMemPool_t ec_pool()
{
	static std::mutex mu;
	static std::map<int, cudaMemPool_t> pools;
	std::lock_guard<std::mutex> lock(mu);
	int dev = 0;

	if (cudaSuccess != cudaGetDevice(&dev))
		return nullptr;

	cudaMemPool_t& p = pools[dev];

	if (nullptr == p) {

		cudaMemPoolProps props = {};
		props.allocType = cudaMemAllocationTypePinned;
		props.location.type = cudaMemLocationTypeDevice;
		props.location.id = dev;

		if (cudaSuccess != cudaMemPoolCreate(&p, &props)) {

			cudaGetLastError();
			p = nullptr;
			return nullptr;
		}

		unsigned long long keep = ~0ull;
		cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
	}

	return p;
}

static cudaError_t ec_malloc(void** q, size_t bytes, cudaStream_t st)
{
	cudaMemPool_t p = ec_pool();
	return p ? cudaMallocFromPoolAsync(q, bytes, p, st) : cudaMallocAsync(q, bytes, st);
}

// Hermitian eigen-decomposition of the n x n matrix that the column-major
// view of A shows (for a row-major Hermitian G that is conj(G), what the
// reference hands LAPACK): eigenvalues ascending in w, eigenvector i in
// column i (= row i of the row-major array).
static int ec_heevd(int n, float2* A, float* w, cudaStream_t st)
{
	const EcSolver* api = nullptr;
	TRY(ec_solver(&api));

	// one handle per device and host thread for the life of the process
	// (creating one per call costs more than a small decomposition):
	// calibrations on several threads, each on its own stream, run their
	// decompositions concurrently
	static std::mutex hmu;
	static std::map<std::pair<int, std::thread::id>, cusolverDnHandle_t> handles;
	int dev = 0;
	CUDA_TRY(cudaGetDevice(&dev));
	cusolverDnHandle_t h = nullptr;

	{
		std::lock_guard<std::mutex> lock(hmu);
		cusolverDnHandle_t& slot = handles[std::make_pair(dev, std::this_thread::get_id())];

		if (nullptr == slot && CUSOLVER_STATUS_SUCCESS != api->create(&slot)) {

			slot = nullptr;
			return fail(BNUFFT_ERR_CUDA, "ecalib: cusolverDnCreate failed");
		}

		h = slot;
	}

	int status = BNUFFT_OK;
	int lwork = 0;
	cuComplex* work = nullptr;
	int* info = nullptr;
	int hinfo = 0;
	if (CUSOLVER_STATUS_SUCCESS != api->set_stream(h, st)
	    || CUSOLVER_STATUS_SUCCESS != api->heevd_size(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, (const cuComplex*)A, n, w, &lwork)) {

		status = fail(BNUFFT_ERR_CUDA, "ecalib: cheevd workspace query failed");

	} else if (cudaSuccess != ec_malloc((void**)&work, sizeof(cuComplex) * (size_t)std::max(lwork, 1), st)
		   || cudaSuccess != ec_malloc((void**)&info, sizeof(int), st)) {

		status = fail(BNUFFT_ERR_NOMEM, "ecalib: cheevd workspace (%d) allocation failed", lwork);

	} else if (CUSOLVER_STATUS_SUCCESS != api->heevd(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, (cuComplex*)A, n, w, work, lwork, info)
		   || cudaSuccess != cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, st)
		   || cudaSuccess != cudaStreamSynchronize(st)) {

		status = fail(BNUFFT_ERR_CUDA, "ecalib: cheevd failed");

	} else if (0 != hinfo) {

		status = fail(BNUFFT_ERR_CUDA, "ecalib: cheevd info %d", hinfo);
	}

	if (work)
		cudaFreeAsync(work, st);

	if (info)
		cudaFreeAsync(info, st);

	return status;
}

// fftmod phase of index j on an axis of length n (src/num/fft.c:62-90)
static std::complex<double> ec_fftmod(long n, long j, bool inv)
{
	const long c = n / 2;
	const double ph = ((double)j - (double)c / 2.) * ((double)c / (double)n);
	const double rem = ph - std::floor(ph);
	const double sg = inv ? -1. : 1.;

	if (0. == rem)
		return 1.;

	if (0.5 == rem)
		return -1.;

	if (0.25 == rem)
		return std::complex<double>(0., sg);

	if (0.75 == rem)
		return std::complex<double>(0., -sg);

	return std::polar(1., 2. * M_PI * sg * rem);
}

// The linear map of the reference's sinc_resize along one axis from n to m
// points (src/misc/resize.c:234-261: fftmod, FFT, fftmod, centred
// zero-padding, ifftmod, unnormalised inverse FFT, ifftmod), [m][n]
// row-major.
static std::vector<double2> ec_sinc_matrix(long n, long m)
{
	std::vector<double2> R((size_t)(m * n), make_double2(0., 0.));

	if (n == m) {

		for (long i = 0; i < n; i++)
			R[(size_t)(i * n + i)] = make_double2(1., 0.);

		return R;
	}

	const long p = m / 2 - n / 2;
	std::vector<std::complex<double>> em((size_t)m), en((size_t)n), pm((size_t)m), pn((size_t)n), a((size_t)n);

	for (long k = 0; k < m; k++) {

		em[(size_t)k] = std::polar(1., 2. * M_PI * (double)k / (double)m);
		pm[(size_t)k] = ec_fftmod(m, k, true);
	}

	for (long k = 0; k < n; k++) {

		en[(size_t)k] = std::polar(1., -2. * M_PI * (double)k / (double)n);
		pn[(size_t)k] = ec_fftmod(n, k, false);
	}

	for (long u = 0; u < n; u++) {

		for (long f = 0; f < n; f++)		// forward half: fftmod, DFT, fftmod
			a[(size_t)f] = pn[(size_t)f] * en[(size_t)(f * u % n)] * pn[(size_t)u];

		for (long x = 0; x < m; x++) {		// centred padding, ifftmod, inverse DFT, ifftmod

			std::complex<double> s = 0.;

			for (long f = 0; f < n; f++) {

				const long g = f + p;
				s += em[(size_t)(g * x % m)] * pm[(size_t)g] * a[(size_t)f];
			}

			s *= pm[(size_t)x];
			R[(size_t)(x * n + u)] = make_double2(s.real(), s.imag());
		}
	}

	return R;
}

// The kernel-image transform: zero-pad [kx, ky, kz] centred into
// [xh, yh, zh], ifftmod, unnormalised inverse FFT (src/calib/calib.c
// :1004-1057), as a [hd][kd] row-major matrix.
static std::vector<float2> ec_kernel_dft(const long kd3[3], const long hd3[3])
{
	const long kd = kd3[0] * kd3[1] * kd3[2], hd = hd3[0] * hd3[1] * hd3[2];
	std::vector<std::complex<double>> ax[3];

	for (int a = 0; a < 3; a++) {

		const long h = hd3[a], k = kd3[a], p = h / 2 - k / 2;
		ax[a].resize((size_t)(h * k));

		for (long x = 0; x < h; x++)
			for (long u = 0; u < k; u++)
				ax[a][(size_t)(x * k + u)] = std::polar(1., 2. * M_PI * (double)((u + p) * x % h) / (double)h) * ec_fftmod(h, u + p, true);
	}

	std::vector<float2> F((size_t)(hd * kd));

	for (long x = 0; x < hd; x++)
		for (long u = 0; u < kd; u++) {

			const long x0 = x % hd3[0], x1 = (x / hd3[0]) % hd3[1], x2 = x / (hd3[0] * hd3[1]);
			const long u0 = u % kd3[0], u1 = (u / kd3[0]) % kd3[1], u2 = u / (kd3[0] * kd3[1]);
			const std::complex<double> v = ax[0][(size_t)(x0 * kd3[0] + u0)] * ax[1][(size_t)(x1 * kd3[1] + u1)] * ax[2][(size_t)(x2 * kd3[2] + u2)];
			F[(size_t)(x * kd + u)] = make_float2((float)v.real(), (float)v.imag());
		}

	return F;
}

// The calibration region (src/misc/mri2.c:100-160): inside the centre
// block td (per-voxel coil energies e, host copy), grow a centred fully
// sampled block one line at a time per dimension up to calsize, then slide
// along the readout to the position of largest energy (first maximum).
static void ec_calib_geom(const std::vector<float>& e, const long td[3], const long calsize[3], long cal[3], long pos[3])
{
	for (int i = 0; i < 3; i++) {

		cal[i] = 1;
		pos[i] = (td[i] - 1) / 2;
	}

	bool stop[3] = { false, false, false };

	auto full = [&]() {

		for (long z = 0; z < cal[2]; z++)
			for (long y = 0; y < cal[1]; y++)
				for (long x = 0; x < cal[0]; x++)
					if (0.f == e[(size_t)((pos[0] + x) + td[0] * ((pos[1] + y) + td[1] * (pos[2] + z)))])
						return false;
		return true;
	};

	while (!(stop[0] && stop[1] && stop[2])) {

		for (int i = 0; i < 3; i++) {

			if (cal[i] == td[i] || cal[i] >= calsize[i])
				stop[i] = true;

			if (stop[i])
				continue;

			cal[i]++;
			pos[i] = (td[i] - cal[i]) / 2;

			if (!full()) {

				cal[i]--;
				pos[i] = (td[i] - cal[i]) / 2;
				stop[i] = true;
			}
		}
	}

	// readout sweep: energy of every readout line inside the y/z window,
	// then window sums by a running sum
	std::vector<double> line((size_t)td[0], 0.);

	for (long z = 0; z < cal[2]; z++)
		for (long y = 0; y < cal[1]; y++)
			for (long x = 0; x < td[0]; x++)
				line[(size_t)x] += e[(size_t)(x + td[0] * ((pos[1] + y) + td[1] * (pos[2] + z)))];

	long best = 0;
	double beng = 0., win = 0.;

	for (long x = 0; x < cal[0]; x++)
		win += line[(size_t)x];

	for (long r = 0; r + cal[0] <= td[0]; r++) {

		if (r > 0)
			win += line[(size_t)(r + cal[0] - 1)] - line[(size_t)(r - 1)];

		if (std::sqrt(std::max(win, 0.)) > beng) {

			best = r;
			beng = std::sqrt(std::max(win, 0.));
		}
	}

	pos[0] = best;
}

struct EcBuf {

	cudaStream_t st;
	std::vector<void*> p;
	explicit EcBuf(cudaStream_t s) : st(s) {}
	~EcBuf() { for (void* q : p) cudaFreeAsync(q, st); }

	template <class T>
	int alloc(T** out, size_t n)
	{
		void* q = nullptr;

		if (cudaSuccess != ec_malloc(&q, std::max<size_t>(n, 1) * sizeof(T), st)) {

			cudaGetLastError();
			return fail(BNUFFT_ERR_NOMEM, "ecalib: out of device memory (%zu bytes)", n * sizeof(T));
		}

		p.push_back(q);
		*out = (T*)q;
		return BNUFFT_OK;
	}
};

template <int W>
static int ec_launch_eigen(int X, int Y, int Z, int C, int M, int xh, int L, const double2* T, const double2* Rx,
			   const float2* rot, int iters, float crop, int soft, int intensity, float2* sens, float2* ev, cudaStream_t st)
{
	constexpr int PX = 8 * 32 / W;
	const int mmax = (M <= 4) ? 4 : 8;
	const size_t smem = sizeof(double2) * ((size_t)xh * L + (size_t)PX * xh) + sizeof(float2) * (size_t)(8 * 32 * mmax)
			    + sizeof(float2) * (size_t)PX * M * C + sizeof(float) * PX * M;

	auto kern = (M <= 4) ? bn::k_ec_eigen<W, 4> : bn::k_ec_eigen<W, 8>;

	if (smem > 200 * 1024)		// the opt-in prep_kernel sets, once per kernel and device
		return fail(BNUFFT_ERR_UNSUPPORTED, "ecalib: %d coils with a %d-point kernel grid need %zu bytes of shared memory", C, xh, smem);

	TRY(prep_kernel(kern, smem));

	dim3 grid((unsigned)(Y * Z), (unsigned)((X + PX - 1) / PX));
	cudaEvent_t pe = prof_begin("ecalib_pixels", st);
	kern<<<grid, 256, smem, st>>>(X, Y, Z, C, M, xh, L, T, Rx, rot, iters, crop, soft, intensity, sens, ev);
	prof_end(pe, st);
	LAUNCHED();
	return BNUFFT_OK;
}

static unsigned ec_blocks(long n) { return (unsigned)std::min<long>((n + 255) / 256, 148L * 16); }

// mode 0: A B; 1: A^H B (the Gram A^H A); 2: A B^H (A A^H); the two Gram
// modes compute the lower triangle only (see k_ec_cgemm)
static int ec_gemm(int mode, int M, int N, int K, const float2* A, long lda, const float2* B, long ldb, float2* Cm, long ldc, cudaStream_t st)
{
	dim3 grid((unsigned)((N + 63) / 64), (unsigned)((M + 63) / 64));

	if (1 == mode)
		bn::k_ec_cgemm<true, false, true><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, Cm, ldc);
	else if (2 == mode)
		bn::k_ec_cgemm<false, true, true><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, Cm, ldc);
	else
		bn::k_ec_cgemm<false, false><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, Cm, ldc);

	LAUNCHED();
	return BNUFFT_OK;
}

extern "C" void bnufft_ecalib_defaults(struct bnufft_ecalib_conf* conf)
{
	for (int i = 0; i < 3; i++) {

		conf->kdims[i] = 6;
		conf->calsize[i] = 24;
	}

	conf->maps = 2;
	conf->threshold = 0.001f;
	conf->numsv = -1;
	conf->percentsv = -1.f;
	conf->crop = 0.8f;
	conf->softcrop = 0;
	conf->rotphase = 1;
	conf->orthiter = 1;
	conf->num_orthiter = 30;
	conf->weighting = 0;
	conf->intensity = 0;
	conf->phase_normalize = 0;
	conf->nystroem = 0;
}

extern "C" int bnufft_ecalib_dims(const struct bnufft_ecalib_conf* conf, int N, const long ksp_dims[], long sens_dims[], long emaps_dims[])
{
	if (nullptr == conf || N < 5 || nullptr == ksp_dims)
		return fail(BNUFFT_ERR_ARG, "ecalib: bad arguments");

	for (int i = 0; i < N; i++) {

		if (nullptr != sens_dims)
			sens_dims[i] = 1;

		if (nullptr != emaps_dims)
			emaps_dims[i] = 1;
	}

	for (int i = 0; i < 3; i++) {

		const long k = (1 == ksp_dims[i]) ? 1 : conf->kdims[i];

		if (nullptr != sens_dims)
			sens_dims[i] = (k > 1) ? ksp_dims[i] : 1;

		if (nullptr != emaps_dims)
			emaps_dims[i] = (k > 1) ? ksp_dims[i] : 1;
	}

	if (nullptr != sens_dims) {

		sens_dims[3] = ksp_dims[3];
		sens_dims[4] = conf->maps;
	}

	if (nullptr != emaps_dims)
		emaps_dims[4] = conf->maps;

	return BNUFFT_OK;
}

// the options and sizes this build implements (src/ecalib.c:64-97)
static int ec_check(const struct bnufft_ecalib_conf* conf, long C, int M)
{
	if (conf->weighting || conf->phase_normalize || conf->nystroem || !conf->orthiter || conf->crop < 0.f)
		return fail(BNUFFT_ERR_UNSUPPORTED, "ecalib: soft-weighting, automatic (SURE) crop, phase normalisation, "
			    "Nystroem and the full point-wise eigen-decomposition are not built");

	if (C < 1)
		return fail(BNUFFT_ERR_ARG, "ecalib: no coils");

	if (C > 32)
		return fail(BNUFFT_ERR_UNSUPPORTED, "ecalib: %ld coils (at most 32 are built)", C);

	if (M < 1 || M > C || M > 8)
		return fail(BNUFFT_ERR_ARG, "ecalib: %d maps for %ld coils (1 <= maps <= min(coils, 8))", M, C);

	return BNUFFT_OK;
}

// Steps 2-7 from the calibration data on the device (cal [cx, cy, cz, C]):
// the Gram matrix of the Casorati matrix, its eigen-decomposition, the
// kernels, their images and per-pixel Gram matrices, the interpolation and
// the per-pixel pass into sens [od, C, M] and emaps [od, 1, M].
// cov_out (not NULL): stop after step 4 and write the low-resolution
// covariance there in the reference's calone layout [xh, yh, zh, C(C+1)/2]
// (the pixel index fastest; host or device memory).
static int ec_from_calibration(const struct bnufft_ecalib_conf* conf, const long kd3[3], const long od[3], long C, int M,
			       const float2* dcal, const long cal[3], float* svals, long* nkernels, void* sens, void* emaps,
			       cudaStream_t st, EcBuf& buf, void* cov_out = nullptr)
{
	using namespace bn;

	const long csize = cal[0] * cal[1] * cal[2];

	// 2. Casorati matrix and its Gram matrix G = A^H A (row-major)
	const long kd = kd3[0] * kd3[1] * kd3[2];
	const long Ncol = kd * C;
	const long P = (cal[0] - kd3[0] + 1) * (cal[1] - kd3[1] + 1) * (cal[2] - kd3[2] + 1);

	if (Ncol > 16384)
		return fail(BNUFFT_ERR_UNSUPPORTED, "ecalib: calibration matrix with %ld columns", Ncol);

	// With fewer patches than kernel entries (2D with 11 coils or more) the
	// P x P matrix A A^H has the same nonzero eigenvalues and a smaller
	// decomposition; the kernels follow from its eigenvectors (step 4).
	const bool left = P < Ncol;
	const long R = left ? P : Ncol;
	float2 *dA = nullptr, *dG = nullptr;
	float* dw = nullptr;
	TRY(buf.alloc(&dA, (size_t)(P * Ncol)));
	TRY(buf.alloc(&dG, (size_t)(R * R)));
	TRY(buf.alloc(&dw, (size_t)R));
	cudaEvent_t pe = prof_begin("ecalib_gram", st);
	k_ec_casorati<<<ec_blocks(P * Ncol), 256, 0, st>>>(dcal, (int)cal[0], (int)cal[1], (int)cal[2], (int)kd3[0], (int)kd3[1], (int)kd3[2], (int)C, dA);
	LAUNCHED();

	if (left)
		TRY(ec_gemm(2, (int)P, (int)P, (int)Ncol, dA, Ncol, dA, Ncol, dG, P, st));
	else
		TRY(ec_gemm(1, (int)Ncol, (int)Ncol, (int)P, dA, Ncol, dA, Ncol, dG, Ncol, st));

	prof_end(pe, st);

	// 3. eigen-decomposition of the matrix the column-major view shows:
	// conj(G) as LAPACK sees the reference's row-major array, or conj(A A^H)
	// whose eigenvectors give conj(G)'s through A; kernels above the
	// threshold
	pe = prof_begin("ecalib_eig", st);
	TRY(ec_heevd((int)R, dG, dw, st));
	prof_end(pe, st);
	std::vector<float> w((size_t)R);
	CUDA_TRY(cudaMemcpyAsync(w.data(), dw, sizeof(float) * R, cudaMemcpyDeviceToHost, st));
	CUDA_TRY(cudaStreamSynchronize(st));

	std::vector<float> val((size_t)Ncol, 0.f);

	for (long i = 0; i < R; i++) {

		const float e = w[(size_t)(R - 1 - i)];
		val[(size_t)i] = (e < 0.f) ? 0.f : sqrtf(e);
	}

	if (val[0] <= 0.f)
		return fail(BNUFFT_ERR_ARG, "ecalib: No signal.");

	long n = 0;

	if (-1 != conf->numsv)
		n = conf->numsv;
	else if (-1.f != conf->percentsv)
		n = (long)((float)Ncol * conf->percentsv / 100.f);
	else
		for (long i = 0; i < Ncol; i++)
			if (val[(size_t)i] / val[0] > sqrtf(conf->threshold))
				n++;

	if (n < 1 || n > R || val[(size_t)(n - 1)] <= 0.f)
		return fail(BNUFFT_ERR_ARG, "ecalib: %ld kernels selected (of %ld, rank at most %ld)", n, Ncol, R);

	if (nullptr != svals)
		for (long i = 0; i < Ncol; i++)
			svals[i] = val[(size_t)i];

	if (nullptr != nkernels)
		*nkernels = n;

	// 4. kernel images on the (2k)^d grid and their per-pixel Gram matrices
	const long hd3[3] = { kd3[0] > 1 ? 2 * kd3[0] : 1, kd3[1] > 1 ? 2 * kd3[1] : 1, kd3[2] > 1 ? 2 * kd3[2] : 1 };
	const long hd = hd3[0] * hd3[1] * hd3[2];
	const long L = C * (C + 1) / 2;
	float2 *dKT = nullptr, *dF = nullptr, *dKimg = nullptr;
	double2* dcov = nullptr;
	TRY(buf.alloc(&dKT, (size_t)(kd * C * n)));
	TRY(buf.alloc(&dF, (size_t)(hd * kd)));
	TRY(buf.alloc(&dKimg, (size_t)(hd * C * n)));
	TRY(buf.alloc(&dcov, (size_t)(hd * L)));
	const std::vector<float2> F = ec_kernel_dft(kd3, hd3);
	CUDA_TRY(cudaMemcpyAsync(dF, F.data(), sizeof(float2) * F.size(), cudaMemcpyHostToDevice, st));
	float* dinv = nullptr;

	if (left) {

		std::vector<float> inv((size_t)n);

		for (long i = 0; i < n; i++)
			inv[(size_t)i] = 1.f / val[(size_t)i];

		TRY(buf.alloc(&dinv, (size_t)n));
		CUDA_TRY(cudaMemcpyAsync(dinv, inv.data(), sizeof(float) * n, cudaMemcpyHostToDevice, st));
	}

	pe = prof_begin("ecalib_imgcov", st);

	if (left)
		k_ec_kern_left<<<ec_blocks(kd * C * n), 256, 0, st>>>(dA, dG, (int)P, (int)Ncol, (int)kd, (int)C, (int)n, dinv, dKT);
	else
		k_ec_kern_perm<<<ec_blocks(kd * C * n), 256, 0, st>>>(dG, (int)Ncol, (int)kd, (int)C, (int)n, dKT);

	LAUNCHED();
	TRY(ec_gemm(0, (int)hd, (int)(C * n), (int)kd, dF, kd, dKT, C * n, dKimg, C * n, st));
	const double scale = 1. / ((double)kd * (double)hd);
	k_ec_pixgram<<<(unsigned)hd, 256, 0, st>>>(dKimg, (int)C, (int)n, scale, dcov);
	LAUNCHED();
	prof_end(pe, st);

	if (nullptr != cov_out) {

		float2* dout = (float2*)cov_out;
		const bool odev = on_device(cov_out);

		if (!odev)
			TRY(buf.alloc(&dout, (size_t)(hd * L)));

		k_ec_cov_layout<<<ec_blocks(hd * L), 256, 0, st>>>(dcov, hd, L, dout);
		LAUNCHED();

		if (!odev)
			CUDA_TRY(cudaMemcpyAsync(cov_out, dout, sizeof(float2) * hd * L, cudaMemcpyDeviceToHost, st));

		CUDA_TRY(cudaStreamSynchronize(st));
		return BNUFFT_OK;
	}

	// 5. sinc interpolation along y and z to every image row
	const std::vector<double2> Rx = ec_sinc_matrix(hd3[0], od[0]);
	const std::vector<double2> Ry = ec_sinc_matrix(hd3[1], od[1]);
	const std::vector<double2> Rz = ec_sinc_matrix(hd3[2], od[2]);
	double2 *dRx = nullptr, *dRy = nullptr, *dRz = nullptr, *dT = nullptr;
	float2* drot = nullptr;
	TRY(buf.alloc(&dRx, Rx.size()));
	TRY(buf.alloc(&dRy, Ry.size()));
	TRY(buf.alloc(&dRz, Rz.size()));
	TRY(buf.alloc(&dT, (size_t)(od[1] * od[2] * hd3[0] * L)));
	TRY(buf.alloc(&drot, (size_t)C));
	CUDA_TRY(cudaMemcpyAsync(dRx, Rx.data(), sizeof(double2) * Rx.size(), cudaMemcpyHostToDevice, st));
	CUDA_TRY(cudaMemcpyAsync(dRy, Ry.data(), sizeof(double2) * Ry.size(), cudaMemcpyHostToDevice, st));
	CUDA_TRY(cudaMemcpyAsync(dRz, Rz.data(), sizeof(double2) * Rz.size(), cudaMemcpyHostToDevice, st));
	pe = prof_begin("ecalib_interp", st);
	k_ec_interp_yz<<<(unsigned)(od[1] * od[2]), 256, 0, st>>>(dcov, (int)hd3[0], (int)hd3[1], (int)hd3[2], (int)L, (int)od[1], dRy, dRz, dT);
	prof_end(pe, st);
	LAUNCHED();

	// 6. phase reference: first principal coil component of the
	// calibration data (src/calib/cc.c:45-62), last component real >= 0
	std::vector<float2> rot((size_t)C, make_float2(0.f, 0.f));

	if (conf->rotphase) {

		float2* dGc = nullptr;
		float* dwc = nullptr;
		TRY(buf.alloc(&dGc, (size_t)(C * C)));
		TRY(buf.alloc(&dwc, (size_t)C));
		k_ec_coilcov<<<(unsigned)(C * C), 256, 0, st>>>(dcal, csize, (int)C, dGc);
		LAUNCHED();
		TRY(ec_heevd((int)C, dGc, dwc, st));
		CUDA_TRY(cudaMemcpyAsync(rot.data(), dGc + (C - 1) * C, sizeof(float2) * C, cudaMemcpyDeviceToHost, st));
		CUDA_TRY(cudaStreamSynchronize(st));
		const std::complex<double> last(rot[(size_t)(C - 1)].x, rot[(size_t)(C - 1)].y);

		if (std::abs(last) > 0.) {

			const std::complex<double> f = std::conj(last) / std::abs(last);

			for (long c = 0; c < C; c++) {

				const std::complex<double> r = std::complex<double>(rot[(size_t)c].x, rot[(size_t)c].y) * f;
				rot[(size_t)c] = make_float2((float)r.real(), (float)r.imag());
			}
		}

	} else {

		rot[0] = make_float2(1.f, 0.f);
	}

	CUDA_TRY(cudaMemcpyAsync(drot, rot.data(), sizeof(float2) * C, cudaMemcpyHostToDevice, st));

	// 7. the fused per-pixel pass
	const long npix = od[0] * od[1] * od[2];
	const bool sdev = on_device(sens), edev = (nullptr == emaps) || on_device(emaps);
	float2* dsens = (float2*)sens;
	float2* dev_ev = (float2*)emaps;

	if (!sdev)
		TRY(buf.alloc(&dsens, (size_t)(npix * C * M)));

	if (!edev)
		TRY(buf.alloc(&dev_ev, (size_t)(npix * M)));

	const int W = (C <= 8) ? 8 : (C <= 16) ? 16 : 32;
	auto go = [&](auto w) -> int {
		return ec_launch_eigen<decltype(w)::value>((int)od[0], (int)od[1], (int)od[2], (int)C, M, (int)hd3[0], (int)L, dT, dRx, drot,
							   conf->num_orthiter, conf->crop, conf->softcrop, conf->intensity, dsens, dev_ev, st);
	};

	if (8 == W)
		TRY(go(std::integral_constant<int, 8>()));
	else if (16 == W)
		TRY(go(std::integral_constant<int, 16>()));
	else
		TRY(go(std::integral_constant<int, 32>()));

	if (!sdev)
		CUDA_TRY(cudaMemcpyAsync(sens, dsens, sizeof(float2) * npix * C * M, cudaMemcpyDeviceToHost, st));

	if (!edev)
		CUDA_TRY(cudaMemcpyAsync(emaps, dev_ev, sizeof(float2) * npix * M, cudaMemcpyDeviceToHost, st));

	// the temporaries are freed when this returns: finish the work first
	CUDA_TRY(cudaStreamSynchronize(st));
	return BNUFFT_OK;
}

static int ec_ecalib(const struct bnufft_ecalib_conf* conf, int N, const long ksp_dims[], const void* ksp,
		     void* sens, void* emaps, float* svals, long* nkernels, long caldims[3], void* stream, void* cov_out)
{
	using namespace bn;

	if (nullptr == conf || nullptr == ksp_dims || nullptr == ksp || (nullptr == sens && nullptr == cov_out) || N < 5)
		return fail(BNUFFT_ERR_ARG, "ecalib: bad arguments");

	if (1 != ksp_dims[4])
		return fail(BNUFFT_ERR_ARG, "ecalib: MAPS dimension is not of size one");

	for (int i = 5; i < N; i++)
		if (1 != ksp_dims[i])
			return fail(BNUFFT_ERR_UNSUPPORTED, "ecalib: one calibration at a time (dimension %d has size %ld)", i, ksp_dims[i]);

	const long X = ksp_dims[0], Y = ksp_dims[1], Z = ksp_dims[2], C = ksp_dims[3];
	const int M = conf->maps;

	if (X < 1 || Y < 1 || Z < 1 || C < 1)
		return fail(BNUFFT_ERR_ARG, "ecalib: bad k-space dimensions");

	TRY(ec_check(conf, C, M));

	long kd3[3], od[3];

	for (int i = 0; i < 3; i++) {

		kd3[i] = (1 == ksp_dims[i]) ? 1 : conf->kdims[i];

		if (kd3[i] < 1 || conf->calsize[i] < 1)
			return fail(BNUFFT_ERR_ARG, "ecalib: bad kernel or calibration size");

		od[i] = (kd3[i] > 1) ? ksp_dims[i] : 1;

		if (kd3[i] > 1 && ksp_dims[i] < 2 * kd3[i])
			return fail(BNUFFT_ERR_ARG, "ecalib: image size %ld below twice the kernel size %ld", ksp_dims[i], kd3[i]);
	}

	cudaStream_t st = (cudaStream_t)stream;
	EcBuf buf(st);
	const long nksp = X * Y * Z * C;
	const float2* dksp = (const float2*)ksp;

	if (!on_device(ksp)) {

		float2* t = nullptr;
		TRY(buf.alloc(&t, (size_t)nksp));
		CUDA_TRY(cudaMemcpyAsync(t, ksp, sizeof(float2) * nksp, cudaMemcpyHostToDevice, st));
		dksp = t;
	}

	// 1. coil energies of the centre block (full readout) to the host,
	// calibration region there
	const long td[3] = { X, std::min(conf->calsize[1], Y), std::min(conf->calsize[2], Z) };
	const long tp[3] = { 0, (Y - td[1]) / 2, (Z - td[2]) / 2 };
	const long tn = td[0] * td[1] * td[2];
	float* den = nullptr;
	TRY(buf.alloc(&den, (size_t)tn));
	k_ec_energy<<<ec_blocks(tn), 256, 0, st>>>(dksp, X, Y, Z, (int)C, (int)tp[0], (int)tp[1], (int)tp[2], (int)td[0], (int)td[1], (int)td[2], den);
	LAUNCHED();
	std::vector<float> hen((size_t)tn);
	CUDA_TRY(cudaMemcpyAsync(hen.data(), den, sizeof(float) * tn, cudaMemcpyDeviceToHost, st));
	CUDA_TRY(cudaStreamSynchronize(st));

	long cal[3], cpos[3];
	const long cs3[3] = { conf->calsize[0], conf->calsize[1], conf->calsize[2] };
	ec_calib_geom(hen, td, cs3, cal, cpos);

	for (int i = 0; i < 3; i++) {

		if (1 == cal[i] && 1 != ksp_dims[i])
			return fail(BNUFFT_ERR_ARG, "ecalib: Calibration region not found!");

		if (cal[i] < kd3[i])
			return fail(BNUFFT_ERR_ARG, "ecalib: calibration region %ld smaller than the kernel %ld", cal[i], kd3[i]);
	}

	if (nullptr != caldims)
		for (int i = 0; i < 3; i++)
			caldims[i] = cal[i];

	const long csize = cal[0] * cal[1] * cal[2];
	float2* dcal = nullptr;
	TRY(buf.alloc(&dcal, (size_t)(csize * C)));
	k_ec_gather<<<ec_blocks(csize * C), 256, 0, st>>>(dksp, X, Y, Z, (int)C, (int)(tp[0] + cpos[0]), (int)(tp[1] + cpos[1]), (int)(tp[2] + cpos[2]),
							 (int)cal[0], (int)cal[1], (int)cal[2], dcal);
	LAUNCHED();

	return ec_from_calibration(conf, kd3, od, C, M, dcal, cal, svals, nkernels, sens, emaps, st, buf, cov_out);
}

extern "C" int bnufft_ecalib(const struct bnufft_ecalib_conf* conf, int N, const long ksp_dims[], const void* ksp,
			     void* sens, void* emaps, float* svals, long* nkernels, long caldims[3], void* stream)
{
	if (nullptr == sens)
		return fail(BNUFFT_ERR_ARG, "ecalib: bad arguments");

	return ec_ecalib(conf, N, ksp_dims, ksp, sens, emaps, svals, nkernels, caldims, stream, nullptr);
}

extern "C" int bnufft_calone(const struct bnufft_ecalib_conf* conf, int N, const long ksp_dims[], const void* ksp,
			     void* cov, float* svals, long* nkernels, long caldims[3], void* stream)
{
	if (nullptr == cov)
		return fail(BNUFFT_ERR_ARG, "calone: bad arguments");

	return ec_ecalib(conf, N, ksp_dims, ksp, nullptr, nullptr, svals, nkernels, caldims, stream, cov);
}

extern "C" int bnufft_calib(const struct bnufft_ecalib_conf* conf, int N, const long out_dims[], void* sens, void* emaps,
			    int SN, float* svals, const long cal_dims[], const void* cal, void* stream)
{
	using namespace bn;

	if (nullptr == conf || nullptr == out_dims || nullptr == cal_dims || nullptr == cal || nullptr == sens || N < 5)
		return fail(BNUFFT_ERR_ARG, "calib: bad arguments");

	for (int i = 5; i < N; i++)
		if (1 != out_dims[i] || 1 != cal_dims[i])
			return fail(BNUFFT_ERR_UNSUPPORTED, "calib: one calibration at a time (dimension %d)", i);

	const long C = cal_dims[3];
	const int M = (int)out_dims[4];

	if (1 != cal_dims[4] || out_dims[3] != C)
		return fail(BNUFFT_ERR_ARG, "calib: output coils %ld, calibration coils %ld", out_dims[3], C);

	TRY(ec_check(conf, C, M));

	long kd3[3], od[3], calv[3];

	for (int i = 0; i < 3; i++) {

		calv[i] = cal_dims[i];
		kd3[i] = (1 == cal_dims[i]) ? 1 : conf->kdims[i];
		od[i] = out_dims[i];

		if (kd3[i] < 1 || calv[i] < kd3[i])
			return fail(BNUFFT_ERR_ARG, "calib: calibration region %ld smaller than the kernel %ld", calv[i], kd3[i]);

		if (od[i] < ((kd3[i] > 1) ? 2 * kd3[i] : 1))
			return fail(BNUFFT_ERR_ARG, "calib: image size %ld below twice the kernel size %ld", od[i], kd3[i]);
	}

	if (nullptr != svals && SN < kd3[0] * kd3[1] * kd3[2] * C)
		return fail(BNUFFT_ERR_ARG, "calib: %d singular values for a %ld-column calibration matrix", SN, kd3[0] * kd3[1] * kd3[2] * C);

	cudaStream_t st = (cudaStream_t)stream;
	EcBuf buf(st);
	const long n = calv[0] * calv[1] * calv[2] * C;
	const float2* dcal = (const float2*)cal;

	if (!on_device(cal)) {

		float2* t = nullptr;
		TRY(buf.alloc(&t, (size_t)n));
		CUDA_TRY(cudaMemcpyAsync(t, cal, sizeof(float2) * n, cudaMemcpyHostToDevice, st));
		dcal = t;
	}

	long nk = 0;
	return ec_from_calibration(conf, kd3, od, C, M, dcal, calv, svals, &nk, sens, emaps, st, buf);
}
