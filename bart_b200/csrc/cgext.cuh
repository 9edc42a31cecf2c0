// CG with the library's fused vector passes for an operator the caller
// applies between the calls (include/bnufft.h, bnufft_cg_*): e.g. the coil
// share of A^H A on each GPU followed by an all-reduce of the result. The
// scalars (rs, alpha, beta, the stopping test) stay on the device in
// float64 as in the one-GPU solve; the iteration is
//
//   q = A p (caller)                 -> bnufft_cg_update: <p, q + lambda p>,
//                                       x += alpha p, r -= alpha (q + lambda p),
//                                       partial ||r||^2        (2 launches)
//   [z = M r (caller, for PCG)]      -> bnufft_cg_direction: beta, p = r + beta p
//                                       (or z + beta p)       (1 or 2 launches)
//
// the reference's conjgrad (src/iter/italgos.c:497-572), its float32
// scalars optionally (cg_keep / cg_ratio). Included into bnufft.cu; uses
// its helpers.

#include <new>

namespace bn {

// per-block partial sums of Re <u, v> = sum Re(conj(u) v) and, if uu_part,
// of ||u||^2
__global__ void k_cgx_dots(const float2* __restrict__ u, const float2* __restrict__ v, long n, double* __restrict__ uv_part,
			   double* __restrict__ uu_part)
{
	__shared__ double sh[32];
	double a = 0., b = 0.;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		const float2 x = u[i], y = v[i];
		a += (double)x.x * y.x + (double)x.y * y.y;
		b += (double)x.x * x.x + (double)x.y * x.y;
	}

	const double sa = block_sum(a, sh);

	if (0 == threadIdx.x)
		uv_part[blockIdx.x] = sa;

	if (uu_part) {

		__syncthreads();
		const double sb = block_sum(b, sh);

		if (0 == threadIdx.x)
			uu_part[blockIdx.x] = sb;
	}
}

// start from x = 0: r = b, p = z (or b); partials of ||b||^2 and <b, z>
__global__ void k_cgx_init(float2* __restrict__ x, float2* __restrict__ r, float2* __restrict__ p, const float2* __restrict__ b,
			   const float2* __restrict__ z, long n, double* __restrict__ bb_part, double* __restrict__ bz_part)
{
	__shared__ double sh[32];
	double a = 0., c = 0.;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		const float2 v = b[i];
		const float2 w = z ? z[i] : v;
		x[i] = make_float2(0.f, 0.f);
		r[i] = v;
		p[i] = w;
		a += (double)v.x * v.x + (double)v.y * v.y;
		c += (double)v.x * w.x + (double)v.y * w.y;
	}

	const double sa = block_sum(a, sh);

	if (0 == threadIdx.x)
		bb_part[blockIdx.x] = sa;

	__syncthreads();
	const double sc = block_sum(c, sh);

	if (0 == threadIdx.x)
		bz_part[blockIdx.x] = sc;
}

// rs[0] = <b, z> (= ||b||^2 without a preconditioner), b2 = ||b||^2,
// eps2 = (tol ||b||)^2 as k_cg_start computes it, done if b = 0
__global__ void k_cgx_start(CgScalars* st, const double* bb_part, const double* bz_part, int nparts, float tol, int f32)
{
	__shared__ double sh[32];
	const double b2 = sum_partials(bb_part, nparts, sh);
	__syncthreads();
	const double bz = sum_partials(bz_part, nparts, sh);

	if (0 == threadIdx.x) {

		st->f32 = f32;
		st->b2 = b2;
		st->rs[0] = cg_keep(st, bz);

		if (f32) {

			float eps = __fmul_rn((float)sqrt(b2), tol);
			st->eps2 = (double)(float)((double)eps * (double)eps);

		} else {

			double eps = (double)tol * sqrt(b2);
			st->eps2 = eps * eps;
		}

		st->iters = 0;
		st->it = 0;
		st->done = (0. == b2);
		st->rnorm = (float)sqrt(b2);
	}
}

// preconditioned direction: rz_new = <r, z> from its partials, the stopping
// test on ||r||^2 (the update's partials), beta = rz_new / rz_old,
// p = z + beta p
__global__ void k_cgx_pdir(float2* __restrict__ p, const float2* __restrict__ z, long n, CgScalars* st, int it,
			   const double* __restrict__ rz_part, int nrz, const double* __restrict__ rr_part, int nrr)
{
	__shared__ double sh[32];

	if (st->done)
		return;

	const double rz_new = cg_keep(st, sum_partials(rz_part, nrz, sh));
	__syncthreads();
	const double rr = sum_partials(rr_part, nrr, sh);
	const double rz_old = st->rs[it & 1];
	const bool stop = (rr <= st->eps2);

	if (!stop) {

		const float beta = cg_ratio(st, rz_new, rz_old);

		for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

			float2 pv = p[i];
			const float2 zv = z[i];
			pv.x = fmaf(beta, pv.x, zv.x);
			pv.y = fmaf(beta, pv.y, zv.y);
			p[i] = pv;
		}
	}

	if ((0 == blockIdx.x) && (0 == threadIdx.x)) {

		st->rs[(it + 1) & 1] = rz_new;
		st->iters = it + 1;
		st->rnorm = (float)sqrt(rr);

		if (stop)
			st->done = 1;
	}
}

}	// namespace bn

struct bnufft_cg_s {

	long n;
	float lam;
	float tol;
	int f32;
	int it;
	int nb;
	bn::CgScalars* st;
	double* part;		// 4 x nb partial sums
};

static int cgx_device(const void* p)
{
	return (nullptr == p) || on_device(p);
}

extern "C" int bnufft_cg_create(bnufft_cg_t* h, long n, float lambda, float tol, int f32_scalars, void* stream)
{
	(void)stream;

	if (nullptr == h || n < 1 || lambda < 0.f || tol < 0.f)
		return fail(BNUFFT_ERR_ARG, "cg_create: bad arguments");

	auto* c = new (std::nothrow) bnufft_cg_s();

	if (nullptr == c)
		return fail(BNUFFT_ERR_NOMEM, "cg_create: out of memory");

	c->n = n;
	c->lam = lambda;
	c->tol = tol;
	c->f32 = f32_scalars ? 1 : 0;
	c->it = 0;
	c->nb = (int)vec_blocks(n);

	if (cudaSuccess != cudaMalloc(&c->st, sizeof(bn::CgScalars))
	    || cudaSuccess != cudaMalloc(&c->part, sizeof(double) * 4 * (size_t)c->nb)) {

		cudaGetLastError();
		cudaFree(c->st);
		delete c;
		return fail(BNUFFT_ERR_NOMEM, "cg_create: out of device memory");
	}

	*h = c;
	return BNUFFT_OK;
}

extern "C" int bnufft_cg_start(bnufft_cg_t c, void* x, void* r, void* p, const void* b, const void* z, void* stream)
{
	using namespace bn;

	if (nullptr == c || nullptr == x || nullptr == r || nullptr == p || nullptr == b)
		return fail(BNUFFT_ERR_ARG, "cg_start: bad arguments");

	if (!(cgx_device(x) && cgx_device(r) && cgx_device(p) && cgx_device(b) && cgx_device(z)))
		return fail(BNUFFT_ERR_ARG, "cg_start: vectors must be device memory");

	cudaStream_t st = S(stream);
	c->it = 0;
	k_cgx_init<<<c->nb, RED_THREADS, 0, st>>>((float2*)x, (float2*)r, (float2*)p, (const float2*)b, (const float2*)z, c->n,
						   c->part, c->part + c->nb);
	LAUNCHED();
	k_cgx_start<<<1, RED_THREADS, 0, st>>>(c->st, c->part, c->part + c->nb, c->nb, c->tol, c->f32);
	LAUNCHED();
	return BNUFFT_OK;
}

extern "C" int bnufft_cg_update(bnufft_cg_t c, void* x, void* r, const void* p, const void* q, void* stream)
{
	using namespace bn;

	if (nullptr == c || nullptr == x || nullptr == r || nullptr == p || nullptr == q)
		return fail(BNUFFT_ERR_ARG, "cg_update: bad arguments");

	cudaStream_t st = S(stream);
	double* pq = c->part;
	double* pp = c->part + c->nb;
	double* rr = c->part + 2 * c->nb;
	k_cgx_dots<<<c->nb, RED_THREADS, 0, st>>>((const float2*)p, (const float2*)q, c->n, pq, pp);
	LAUNCHED();
	k_cg_step<<<c->nb, RED_THREADS, 0, st>>>((float2*)x, (float2*)r, (const float2*)p, (const float2*)q, 1, c->n, c->lam,
						  c->st, c->it, pq, c->nb, pp, c->nb, rr, nullptr);
	LAUNCHED();
	return BNUFFT_OK;
}

extern "C" int bnufft_cg_direction(bnufft_cg_t c, void* p, const void* r, const void* z, void* stream)
{
	using namespace bn;

	if (nullptr == c || nullptr == p || nullptr == r)
		return fail(BNUFFT_ERR_ARG, "cg_direction: bad arguments");

	cudaStream_t st = S(stream);
	double* rr = c->part + 2 * c->nb;

	if (nullptr == z) {

		k_cg_dir<<<c->nb, RED_THREADS, 0, st>>>((float2*)p, (const float2*)r, c->n, c->st, c->it, rr, c->nb);
		LAUNCHED();

	} else {

		double* rz = c->part + 3 * c->nb;
		k_cgx_dots<<<c->nb, RED_THREADS, 0, st>>>((const float2*)r, (const float2*)z, c->n, rz, nullptr);
		LAUNCHED();
		k_cgx_pdir<<<c->nb, RED_THREADS, 0, st>>>((float2*)p, (const float2*)z, c->n, c->st, c->it, rz, c->nb, rr, c->nb);
		LAUNCHED();
	}

	c->it++;
	return BNUFFT_OK;
}

extern "C" int bnufft_cg_status(bnufft_cg_t c, int* done, int* iters, float* rnorm, void* stream)
{
	if (nullptr == c)
		return fail(BNUFFT_ERR_ARG, "cg_status: bad arguments");

	bn::CgScalars s;
	cudaStream_t st = S(stream);
	CUDA_TRY(cudaMemcpyAsync(&s, c->st, sizeof s, cudaMemcpyDeviceToHost, st));
	CUDA_TRY(cudaStreamSynchronize(st));

	if (done)
		*done = s.done;

	if (iters)
		*iters = s.iters;

	if (rnorm)
		*rnorm = s.rnorm;

	return BNUFFT_OK;
}

extern "C" void bnufft_cg_free(bnufft_cg_t c)
{
	if (nullptr == c)
		return;

	cudaFree(c->st);
	cudaFree(c->part);
	delete c;
}
