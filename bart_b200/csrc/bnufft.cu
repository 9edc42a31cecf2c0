// bnufft host side: plans, pass scheduling and the C ABI (include/bnufft.h).
//
// Built for sm_100a only. Every entry point returns a status code instead of
// aborting (the reference aborts through error(), src/misc/misc.c:95).
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <atomic>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/bnufft.h"
#include "nufft_kernels.cuh"
#include "cg_kernels.cuh"
#include "gridding.cuh"
#include "precnet.cuh"
#include "nudft.cuh"
#include "precond_cluster.cuh"
#include "precnet_tc.cuh"

#include <cudaTypedefs.h>

using namespace bn;

// ----------------------------------------------------------------------------
// errors and launch accounting
// ----------------------------------------------------------------------------

static thread_local std::string g_err;
static std::atomic<long> g_launches{0};

static int fail(int code, const char* fmt, ...)
{
	char buf[512];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(buf, sizeof buf, fmt, ap);
	va_end(ap);
	g_err = buf;
	return code;
}

#define CUDA_TRY(call) do { cudaError_t e_ = (call); if (cudaSuccess != e_) \
	return fail(BNUFFT_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); } while (0)

#define LAUNCHED() do { g_launches.fetch_add(1, std::memory_order_relaxed); \
	cudaError_t e_ = cudaGetLastError(); if (cudaSuccess != e_) \
	return fail(BNUFFT_ERR_CUDA, "%s:%d launch: %s", __FILE__, __LINE__, cudaGetErrorString(e_)); } while (0)

#define TRY(call) do { int s_ = (call); if (BNUFFT_OK != s_) return s_; } while (0)

// Optional timing of one kernel class (bnufft_prof_start): a pair of CUDA
// events on the launching stream around every launch of that class.
static std::mutex g_prof_mutex;
static std::string g_prof_target;
static std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_prof_events;

static std::atomic<bool> g_prof_active{false};

// passes run for the preconditioner carry this class prefix ("precond_")
static thread_local bool t_prof_precond = false;

static cudaEvent_t prof_begin(const char* kind, cudaStream_t st)
{
	if (!g_prof_active.load(std::memory_order_relaxed))
		return nullptr;

	std::string k = t_prof_precond ? std::string("precond_") + kind : std::string(kind);

	std::lock_guard<std::mutex> lock(g_prof_mutex);

	if (g_prof_target.empty() || (g_prof_target != k))
		return nullptr;

	cudaEvent_t a, b;
	static std::vector<cudaEvent_t> pool;

	if (pool.size() < 2) {

		for (int i = 0; i < 256; i++) {

			cudaEvent_t e;
			cudaEventCreate(&e);
			pool.push_back(e);
		}
	}

	a = pool.back();
	pool.pop_back();
	b = pool.back();
	pool.pop_back();
	cudaEventRecord(a, st);
	g_prof_events.push_back({ a, b });
	return b;
}

static void prof_end(cudaEvent_t e, cudaStream_t st)
{
	if (e)
		cudaEventRecord(e, st);
}

static cudaStream_t S(void* stream) { return (cudaStream_t)stream; }

// scatter variant of the width-6 gridding: 2 = default (output-stationary
// tiles with register accumulation for 3D multi-channel problems, global
// atomics on bin-sorted samples otherwise), 3 = output-stationary tiles
// wherever they apply (BNUFFT_GRIDDING=lines), 1 = global atomics
// (BNUFFT_GRIDDING=atomic), 0 = shared-memory tiles with shared-memory
// atomics (BNUFFT_GRIDDING=tiles)
static int gridding_kind()
{
	const char* e = getenv("BNUFFT_GRIDDING");	// read per plan (cheap), so callers can switch

	if (e && (0 == strcmp(e, "tiles")))
		return 0;

	if (e && (0 == strcmp(e, "atomic")))
		return 1;

	if (e && (0 == strcmp(e, "lines")))
		return 3;

	return 2;
}

// ----------------------------------------------------------------------------
// Kaiser-Bessel table, roll-off and twiddles (host, float64)
// ----------------------------------------------------------------------------

// I0 from its power series (float64-accurate for |x| <= 30)
static double bessel_i0(double x)
{
	x = fabs(x);
	double q = 0.25 * x * x, term = 1., sum = 1.;

	for (int k = 1; k < 500; k++) {

		term *= q / ((double)k * (double)k);
		sum += term;

		if (term < 1e-18 * sum)
			break;
	}

	return sum;
}

// calc_beta (src/noncart/grid.c:516-519); width/os is a float division
static double calc_beta(float os, float width)
{
	double wos = (double)(width / os);
	return M_PI * sqrt(pow(wos * ((double)os - 0.5), 2.) - 0.8);
}

// beta of the KB table: rolloff_correction() initialises it with a float beta
static double kernel_beta(float os, float width) { return (double)(float)calc_beta(os, width); }

// kb_precompute (src/noncart/grid.c:86-97)
static void kb_precompute(double beta, int n, float* table)
{
	double i0b = bessel_i0(beta);

	for (int i = 0; i < n + 1; i++) {

		double x = (double)i / (double)(n - 1) / 2.;
		table[i] = (fabs(x) >= 0.5) ? 0.f : (float)(bessel_i0(beta * sqrt(1. - pow(2. * x, 2.))) / i0b);
	}
}

// ftkb / rolloff / pos (src/noncart/grid.c:100-117, 522-533)
static double ftkb(double beta, double x, double i0b)
{
	double a = beta * beta - pow(M_PI * x, 2.);

	if (0. == a)
		return 1. / i0b;

	return (a > 0) ? (sinh(sqrt(a)) / sqrt(a)) / i0b : (sin(sqrt(-a)) / sqrt(-a)) / i0b;
}

static double rolloff_axis(int d, int i, float os, float width, double beta, double i0b)
{
	if (1 == d)
		return 1.;

	int od = (int)(os * d);
	int oi = i + (od / 2 - d / 2);
	float p = ((float)oi - (float)(od / 2)) / (float)od;

	return 1. / ftkb(beta, (double)p * (double)width, i0b) / (double)width;
}

// host-only views of the tables above (no device work), for checking them
// against the reference's calc_beta / kb_precompute / rolloff
extern "C" double bnufft_calc_beta(float os, float width) { return calc_beta(os, width); }

extern "C" int bnufft_kb_precompute(double beta, int n, float* table)
{
	if ((n < 2) || !table)
		return fail(BNUFFT_ERR_ARG, "kb_precompute: n >= 2 and a table are needed");

	kb_precompute(beta, n, table);
	return BNUFFT_OK;
}

extern "C" int bnufft_rolloff_axis(float os, float width, long n, double* roll)
{
	if ((n < 1) || !roll)
		return fail(BNUFFT_ERR_ARG, "rolloff: n >= 1 and an output are needed");

	double beta = kernel_beta(os, width);
	double i0b = bessel_i0(beta);

	for (long i = 0; i < n; i++)
		roll[i] = rolloff_axis((int)n, (int)i, os, width, beta, i0b);

	return BNUFFT_OK;
}

// ----------------------------------------------------------------------------
// per-device constant tables
// ----------------------------------------------------------------------------

struct DevTables {

	std::map<int, float2*> twiddle;		// L -> exp(-2 pi i m / L)
	std::map<std::pair<float, float>, float*> kb;	// (os, width) -> table
};

static std::mutex g_tab_mutex;
static std::map<int, DevTables> g_tabs;

// lock-free lookup of tables already built: [device][log2 L]
static std::atomic<const float2*> g_tw_fast[64][16];

// exp(-2 pi i m / L), m = 0..L-1, in float64 then float32
static void twiddles_host(int L, float2* h)
{
	for (int m = 0; m < L; m++) {

		double a = -2. * M_PI * (double)m / (double)L;
		h[m] = make_float2((float)cos(a), (float)sin(a));
	}
}

static int get_twiddles(int L, const float2** out)
{
	int dev;
	CUDA_TRY(cudaGetDevice(&dev));
	int lg = 0;

	while ((1 << lg) < L)
		lg++;

	if ((dev >= 0) && (dev < 64) && (lg < 16)) {

		const float2* f = g_tw_fast[dev][lg].load(std::memory_order_acquire);

		if (f) {

			*out = f;
			return BNUFFT_OK;
		}
	}

	std::lock_guard<std::mutex> lock(g_tab_mutex);
	auto& t = g_tabs[dev].twiddle;
	auto it = t.find(L);

	if (it != t.end()) {

		*out = it->second;
		return BNUFFT_OK;
	}

	std::vector<float2> h(L);
	twiddles_host(L, h.data());
	float2* d = nullptr;
	CUDA_TRY(cudaMalloc(&d, sizeof(float2) * L));
	CUDA_TRY(cudaMemcpy(d, h.data(), sizeof(float2) * L, cudaMemcpyHostToDevice));
	t[L] = d;
	*out = d;

	if ((dev >= 0) && (dev < 64) && (lg < 16) && ((1 << lg) == L))
		g_tw_fast[dev][lg].store(d, std::memory_order_release);

	return BNUFFT_OK;
}

static int get_kb_table(float os, float width, const float** out)
{
	int dev;
	CUDA_TRY(cudaGetDevice(&dev));
	std::lock_guard<std::mutex> lock(g_tab_mutex);
	auto& t = g_tabs[dev].kb;
	auto key = std::make_pair(os, width);
	auto it = t.find(key);

	if (it != t.end()) {

		*out = it->second;
		return BNUFFT_OK;
	}

	std::vector<float> h(KB_TABLE_N + 1);
	kb_precompute(kernel_beta(os, width), KB_TABLE_N, h.data());
	float* d = nullptr;
	CUDA_TRY(cudaMalloc(&d, sizeof(float) * (KB_TABLE_N + 1)));
	CUDA_TRY(cudaMemcpy(d, h.data(), sizeof(float) * (KB_TABLE_N + 1), cudaMemcpyHostToDevice));
	t[key] = d;
	*out = d;
	return BNUFFT_OK;
}

// ----------------------------------------------------------------------------
// FFT pass launchers
// ----------------------------------------------------------------------------

// grid lengths with a DFT: powers of two up to 4096, other lengths up to 2048
// (Bluestein on a power-of-two FFT of at most 4096)
static bool supported_len(int L) { return (L >= 2) && ((L <= 2048) || ((L <= 4096) && (0 == (L & (L - 1))))); }

// dynamic shared memory of a column pass (ColLayout) / row pass (RowLayout), twiddles included
static size_t pass_smem(int L, int B) { return sizeof(float2) * (size_t)L * (size_t)(smem_stride(B) + 1); }
static size_t rows_smem(int L, int B) { return sizeof(float2) * ((size_t)B * (size_t)(L + L / 8) + (size_t)L); }

// sequences per block (B in {4, 8, 16}, B * L / 8 threads <= 1024): as many
// as fit, fewer when the launch would have too few blocks to fill the GPU
static int choose_B(int L, long nseq)
{
	int B = std::min(16, 8192 / L);
	int Bmin = std::min(16, std::max(4, 256 / L));	// at least one warp per block

	while ((B > Bmin) && ((nseq + B - 1) / B < 2 * 148))
		B /= 2;

	return B;
}

// opt in to large dynamic shared memory once per kernel and device; kernels
// also hold static shared memory, so every launch site opts in
static std::mutex g_attr_mutex;
static std::map<std::pair<const void*, int>, bool> g_attr_done;
static thread_local std::pair<const void*, int> g_attr_last[8];
static thread_local int g_attr_next = 0;

template <typename K>
static int prep_kernel(K kernel, size_t smem)
{
	(void)smem;
	int dev;
	CUDA_TRY(cudaGetDevice(&dev));
	auto key = std::make_pair((const void*)kernel, dev);

	for (auto& k : g_attr_last)	// per-thread memo of recent kernels
		if (k == key)
			return BNUFFT_OK;

	std::lock_guard<std::mutex> lock(g_attr_mutex);

	if (!g_attr_done.count(key)) {

		CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
		g_attr_done[key] = true;
	}

	g_attr_last[g_attr_next] = key;
	g_attr_next = (g_attr_next + 1) % 8;
	return BNUFFT_OK;
}

template <int L, int B>
static int launch_rows_fwd_LB(const float2* img, const float2* maps, const float* ax, const float* ayz,
		int X, long YZ, long R, float2* out, cudaStream_t st, const int* done, const Dft& d)
{
	const float2* tw;
	TRY(get_twiddles(L, &tw));
	size_t smem = rows_smem(L, B);
	auto kern = (d.n == L) ? k_rows_fwd<L, B, false> : k_rows_fwd<L, B, true>;
	TRY(prep_kernel(kern, smem));
	cudaEvent_t pe = prof_begin("rows_fwd", st);
	kern<<<(unsigned)((R + B - 1) / B), B * L / 8, smem, st>>>(img, maps, ax, ayz, X, YZ, R, out, tw, done, d);
	prof_end(pe, st);
	LAUNCHED();
	return BNUFFT_OK;
}

template <int L, int B, int MODE>
static int launch_cols_LB(const float2* in, long ies, long ios, int n_in, int wrap_in,
		float2* out, long oes, long oos, int n_out, int wrap_out, int W, long O,
		const float2* psf, long pes, long pmod, long pos, const int* done, cudaStream_t st, const Dft& d)
{
	const float2* tw;
	TRY(get_twiddles(L, &tw));
	size_t smem = pass_smem(L, B);

	if ((d.n == L) && cols_double_buffered(MODE, false, L, B))
		smem += sizeof(float2) * (size_t)L * (size_t)smem_stride(B);	// the second exchange buffer

	auto kern = (d.n == L) ? k_cols<L, B, MODE, false> : k_cols<L, B, MODE, true>;
	TRY(prep_kernel(kern, smem));

	if (O > 65535)
		return fail(BNUFFT_ERR_UNSUPPORTED, "column pass with %ld outer sequences", O);

	dim3 grid((unsigned)((W + B - 1) / B), (unsigned)O);
	cudaEvent_t pe = prof_begin((2 == MODE) ? "cols_toeplitz" : ((1 == MODE) ? "cols_inv" : "cols_fwd"), st);
	kern<<<grid, B * L / 8, smem, st>>>(in, ies, ios, n_in, wrap_in, out, oes, oos, n_out, wrap_out,
			W, psf, pes, pmod, pos, tw, done, d);
	prof_end(pe, st);
	LAUNCHED();
	return BNUFFT_OK;
}

template <int L, int B>
static int launch_rows_inv_LB(const float2* in, const float2* maps, const float* ax, const float* ayz,
		int X, long YZ, int C, int cpg, float2* out, const float2* pdot, double* dot_part, const int* done,
		cudaStream_t st, const Dft& d)
{
	const float2* tw;
	TRY(get_twiddles(L, &tw));
	int groups = (C + cpg - 1) / cpg;
	size_t smem = rows_smem(L, B);
	auto kern = (d.n == L) ? k_rows_inv<L, B, false> : k_rows_inv<L, B, true>;
	TRY(prep_kernel(kern, smem));
	dim3 grid((unsigned)((YZ + B - 1) / B), (unsigned)groups);
	cudaEvent_t pe = prof_begin("rows_inv", st);
	kern<<<grid, B * L / 8, smem, st>>>(in, maps, ax, ayz, X, YZ, C, cpg, out, tw, pdot, dot_part, done, d);
	prof_end(pe, st);
	LAUNCHED();
	return BNUFFT_OK;
}

template <int L, int B>
static int launch_rows_fwd_cg_LB(const float2* bvec, const float2* r, const float2* p_prev, float2* p_cur,
		const float2* maps, const float* ax, const float* ayz, int X, long YZ, long R, float2* out,
		CgScalars* stt, int it, const double* rs_part, int nrs, double* pp_part, cudaStream_t st, const Dft& d)
{
	const float2* tw;
	TRY(get_twiddles(L, &tw));
	size_t smem = rows_smem(L, B);
	auto kern = (d.n == L) ? k_rows_fwd_cg<L, B, false> : k_rows_fwd_cg<L, B, true>;
	TRY(prep_kernel(kern, smem));
	cudaEvent_t pe = prof_begin("rows_fwd", st);
	kern<<<(unsigned)((R + B - 1) / B), B * L / 8, smem, st>>>(bvec, r, p_prev, p_cur, maps, ax, ayz,
			X, YZ, R, out, tw, stt, it, rs_part, nrs, pp_part, d);
	prof_end(pe, st);
	LAUNCHED();
	return BNUFFT_OK;
}

// run CALL with compile-time LL (FFT length) and BB (sequences per block)
#define DISPATCH_LB(L, B, CALL) \
	switch (L) { \
	case 16: { constexpr int LL = 16; DISPATCH_B(B, CALL) } \
	case 32: { constexpr int LL = 32; DISPATCH_B(B, CALL) } \
	case 64: { constexpr int LL = 64; DISPATCH_B(B, CALL) } \
	case 128: { constexpr int LL = 128; DISPATCH_B(B, CALL) } \
	case 256: { constexpr int LL = 256; DISPATCH_B(B, CALL) } \
	case 512: { constexpr int LL = 512; DISPATCH_B(B, CALL) } \
	case 1024: { constexpr int LL = 1024; DISPATCH_B(B, CALL) } \
	case 2048: { constexpr int LL = 2048; DISPATCH_B(B, CALL) } \
	case 4096: { constexpr int LL = 4096; DISPATCH_B(B, CALL) } \
	default: return fail(BNUFFT_ERR_UNSUPPORTED, "FFT length %d (powers of two 16..4096 are built)", L); }

#define DISPATCH_B(B, CALL) \
	switch (B) { \
	case 2: { constexpr int BB = 2; if constexpr (LL >= 4096 && BB * LL / 8 <= 1024) return CALL; break; } \
	case 4: { constexpr int BB = 4; if constexpr (BB * LL / 8 <= 1024 && BB * LL / 8 >= 32) return CALL; break; } \
	case 8: { constexpr int BB = 8; if constexpr (BB * LL / 8 <= 1024 && BB * LL / 8 >= 32) return CALL; break; } \
	case 16: { constexpr int BB = 16; if constexpr (BB * LL / 8 <= 1024 && BB * LL / 8 >= 32) return CALL; break; } \
	} \
	return fail(BNUFFT_ERR_ARG, "no FFT pass instance for L=%d B=%d", L, B);

// DFT of logical length n: the power-of-two FFT of length n itself, or
// Bluestein's algorithm on the power-of-two length P >= 2n - 1 with its
// chirp and filter tables (computed once per device and length on the host
// in float64: chirp exp(-i pi (j^2 mod 2n) / n), filters by a float64 FFT)
struct DftTables {

	int P = 0;
	float2 *chirp = nullptr, *bf = nullptr, *bi = nullptr;
};

static std::mutex g_dft_mutex;
static std::map<std::pair<int, int>, DftTables> g_dft;

static void fft_host(std::vector<std::complex<double>>& a)	// in place, forward, unnormalised
{
	const size_t n = a.size();

	for (size_t i = 1, j = 0; i < n; i++) {

		size_t bit = n >> 1;

		for (; j & bit; bit >>= 1)
			j ^= bit;

		j ^= bit;

		if (i < j)
			std::swap(a[i], a[j]);
	}

	for (size_t len = 2; len <= n; len <<= 1) {

		for (size_t i = 0; i < n; i += len) {

			for (size_t k = 0; k < len / 2; k++) {

				double ang = -2. * M_PI * (double)k / (double)len;
				std::complex<double> w(cos(ang), sin(ang));
				std::complex<double> u = a[i + k];
				std::complex<double> v = a[i + k + len / 2] * w;
				a[i + k] = u + v;
				a[i + k + len / 2] = u - v;
			}
		}
	}
}

static int get_dft(int n, Dft* d, int* P)
{
	d->n = n;
	d->chirp = d->bf = d->bi = nullptr;

	if ((n >= 16) && (n <= 4096) && (0 == (n & (n - 1)))) {

		*P = n;
		return BNUFFT_OK;
	}

	int p = 16;

	while (p < 2 * n - 1)
		p *= 2;

	if ((n < 2) || (p > 4096))
		return fail(BNUFFT_ERR_UNSUPPORTED, "DFT length %d (powers of two up to 4096, other lengths up to 2048)", n);

	int dev;
	CUDA_TRY(cudaGetDevice(&dev));
	std::lock_guard<std::mutex> lock(g_dft_mutex);
	DftTables& t = g_dft[std::make_pair(dev, n)];

	if (!t.P) {

		std::vector<std::complex<double>> c(n), bf(p), bi(p);

		for (long j = 0; j < n; j++) {

			double ang = -M_PI * (double)((j * j) % (2L * n)) / (double)n;
			c[j] = std::complex<double>(cos(ang), sin(ang));
		}

		for (long m = -(n - 1); m <= n - 1; m++) {

			const std::complex<double>& cm = c[(m < 0) ? -m : m];	// c_m = c_{-m}
			bf[(m + p) % p] = std::conj(cm);
			bi[(m + p) % p] = cm;
		}

		fft_host(bf);
		fft_host(bi);
		std::vector<float2> hc(n), hf(p), hi(p);

		for (int j = 0; j < n; j++)
			hc[j] = make_float2((float)c[j].real(), (float)c[j].imag());

		for (int j = 0; j < p; j++) {

			hf[j] = make_float2((float)(bf[j].real() / p), (float)(bf[j].imag() / p));
			hi[j] = make_float2((float)(bi[j].real() / p), (float)(bi[j].imag() / p));
		}

		DftTables nt;
		CUDA_TRY(cudaMalloc(&nt.chirp, sizeof(float2) * n));
		CUDA_TRY(cudaMalloc(&nt.bf, sizeof(float2) * p));
		CUDA_TRY(cudaMalloc(&nt.bi, sizeof(float2) * p));
		CUDA_TRY(cudaMemcpy(nt.chirp, hc.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
		CUDA_TRY(cudaMemcpy(nt.bf, hf.data(), sizeof(float2) * p, cudaMemcpyHostToDevice));
		CUDA_TRY(cudaMemcpy(nt.bi, hi.data(), sizeof(float2) * p, cudaMemcpyHostToDevice));
		nt.P = p;
		t = nt;
	}

	d->chirp = t.chirp;
	d->bf = t.bf;
	d->bi = t.bi;
	*P = t.P;
	return BNUFFT_OK;
}

// The passes below take the logical DFT length n (the grid length) and run
// the power-of-two FFT of length P (n itself or Bluestein's)
static int rows_fwd(int n, const float2* img, const float2* maps, const float* ax, const float* ayz,
		int X, long YZ, long R, float2* out, cudaStream_t st, const int* done = nullptr)
{
	Dft d;
	int L;
	TRY(get_dft(n, &d, &L));
	int B = choose_B(L, R);
	DISPATCH_LB(L, B, (launch_rows_fwd_LB<LL, BB>(img, maps, ax, ayz, X, YZ, R, out, st, done, d)));
}

static int cols(int n, int mode, const float2* in, long ies, long ios, int n_in, int wrap_in,
		float2* out, long oes, long oos, int n_out, int wrap_out, int W, long O,
		const float2* psf, long pes, long pmod, long pos, cudaStream_t st, const int* done = nullptr)
{
	Dft d;
	int L;
	TRY(get_dft(n, &d, &L));
	int B = choose_B(L, (long)W * O);

	while ((B > std::max(4, 256 / L)) && (B > W))
		B /= 2;

	// the double-buffered Toeplitz pass: two blocks of 8 sequences per SM
	// overlap one another's barriers (measured faster than one block of 16)
	if ((2 == mode) && (B > 8) && (d.n == L) && cols_double_buffered(2, false, L, 8))
		B = 8;

	if (const char* e = getenv("BNUFFT_COLS_B")) {	// tuning knob: sequences per block (4, 8, 16)

		int b = atoi(e);

		if (((4 == b) || (8 == b) || (16 == b)) && (b * L / 8 <= 1024) && (b * L / 8 >= 32))
			B = b;
	}

	// 512-point Toeplitz columns of several images (coils): the two-stage
	// transform kernel, 16 threads per column (BNUFFT_TOE512=0 keeps the
	// three-stage k_cols, whose 64 threads per column suit the single-image
	// passes better: 30.7 vs 28.5 us per 16-coil launch, but a slower solve
	// when the preconditioner's one image also takes the new kernel)
	if ((2 == mode) && (512 == L) && (d.n == L) && (O >= 4) && (O <= 65535)) {

		const char* e = getenv("BNUFFT_TOE512");

		if (!(e && (0 == strcmp(e, "0")))) {

			const float2* tw;
			TRY(get_twiddles(L, &tw));
			const size_t smem = sizeof(float2) * (size_t)L * (TOE512_B + 1);
			TRY(prep_kernel(k_cols_toe512, smem));
			dim3 grid((unsigned)((W + TOE512_B - 1) / TOE512_B), (unsigned)O);
			cudaEvent_t pe = prof_begin("cols_toeplitz", st);
			k_cols_toe512<<<grid, TOE512_B * 16, smem, st>>>(in, ies, ios, n_in, wrap_in, out, oes, oos, n_out,
					wrap_out, W, psf, pes, pmod, pos, tw, done);
			prof_end(pe, st);
			LAUNCHED();
			return BNUFFT_OK;
		}
	}

	if (0 == mode)
		DISPATCH_LB(L, B, (launch_cols_LB<LL, BB, 0>(in, ies, ios, n_in, wrap_in, out, oes, oos, n_out, wrap_out, W, O, psf, pes, pmod, pos, done, st, d)))
	else if (1 == mode)
		DISPATCH_LB(L, B, (launch_cols_LB<LL, BB, 1>(in, ies, ios, n_in, wrap_in, out, oes, oos, n_out, wrap_out, W, O, psf, pes, pmod, pos, done, st, d)))
	else
		DISPATCH_LB(L, B, (launch_cols_LB<LL, BB, 2>(in, ies, ios, n_in, wrap_in, out, oes, oos, n_out, wrap_out, W, O, psf, pes, pmod, pos, done, st, d)))
}

static int rows_inv(int n, const float2* in, const float2* maps, const float* ax, const float* ayz,
		int X, long YZ, int C, int cpg, float2* out, cudaStream_t st,
		const float2* pdot = nullptr, double* dot_part = nullptr, const int* done = nullptr, int* nblocks = nullptr)
{
	Dft d;
	int L;
	TRY(get_dft(n, &d, &L));
	int groups = (C + cpg - 1) / cpg;
	int B = choose_B(L, YZ * groups);

	if (nblocks)
		*nblocks = (int)(((YZ + B - 1) / B) * groups);

	DISPATCH_LB(L, B, (launch_rows_inv_LB<LL, BB>(in, maps, ax, ayz, X, YZ, C, cpg, out, pdot, dot_part, done, st, d)));
}

static int rows_fwd_cg(int n, const float2* bvec, const float2* r, const float2* p_prev, float2* p_cur,
		const float2* maps, const float* ax, const float* ayz, int X, long YZ, long R, float2* out,
		CgScalars* stt, int it, const double* rs_part, int nrs, double* pp_part, int* nblocks, cudaStream_t st)
{
	Dft d;
	int L;
	TRY(get_dft(n, &d, &L));
	int B = choose_B(L, R);
	*nblocks = (int)((R + B - 1) / B);
	DISPATCH_LB(L, B, (launch_rows_fwd_cg_LB<LL, BB>(bvec, r, p_prev, p_cur, maps, ax, ayz, X, YZ, R, out,
			stt, it, rs_part, nrs, pp_part, st, d)));
}

static unsigned vec_blocks(long n, int threads = RED_THREADS, int maxb = 4 * 148)
{
	long b = (n + threads - 1) / threads;
	return (unsigned)std::max(1L, std::min<long>(b, maxb));
}

// ----------------------------------------------------------------------------
// geometry and the three NUFFT operators on device buffers
// ----------------------------------------------------------------------------

struct Geom {

	int N[3];	// image dims
	int G[3];	// oversampled dims (2N, lround(os N) when chain, or 1)
	int nd;		// number of transformed (non-singleton) axes
	long npix;	// N0*N1*N2
	long gsz;	// G0*G1*G2
	long M;		// samples
	float os, width;
	int periodic;
	int chain = 0;	// os != 2: the reference's chained NUFFT (src/noncart/nufft_chain.c)
};

struct Work {

	float2* grid = nullptr;	// [gsz * C]
	float2* t1 = nullptr;	// [G0 * N1 * N2 * C]
	float2* t2 = nullptr;	// 3D: [G0 * G1 * N2 * C]
	long cap = 0;		// channels the buffers hold
};

// interpolation matrix in CSR form over grid cells (deterministic gridding)
struct Csr {

	long* row_ptr = nullptr;	// [gsz + 1]
	int* col = nullptr;		// [nnz] sample index
	float* val = nullptr;		// [nnz] weight
	long nnz = 0;
};

// samples sorted by bin of the oversampled grid, cut into sub-blocks
struct Bins {

	BinGeom bg;
	int* perm = nullptr;		// [M] sorted position -> sample index
	float4* traj = nullptr;		// [M] trajectory in sorted order
	int* sub_bin = nullptr;
	int* sub_first = nullptr;
	int* sub_count = nullptr;
	int* sub_start = nullptr;	// [nbins + 1]; sub_start[nbins] = number of sub-blocks
	const int* nsub_dev = nullptr;
	int nsub = 0;			// upper bound of sub-blocks (launch size)
	int cc = 1;			// coil tiles held in shared memory at once
	// output-stationary scatter (k_grid6_tiles): bins are its tiles
	int tg_cfg = -1;		// kernel shape (TG_*), -1: not used
	long ntiles = 0;
	int* bin_start = nullptr;	// [nbins + 1]
	int* work_tile = nullptr;	// [nwork_max]
	int* work_chunk = nullptr;
	int* work_start = nullptr;	// [ntiles + 1]; work_start[ntiles] = work items
	unsigned char* multi = nullptr;	// [ntiles]
	long nwork_max = 0;		// upper bound of work items (launch size)
	int cand = 512;			// candidates per work item
	float4* foot = nullptr;		// [M][FOOT_F4] footprints of the sorted samples
	float2* kperm = nullptr;	// [M][kperm_c] k-space in bin order (large problems)
	long kperm_c = 0;
};

// shapes of k_grid6_tiles <TX, LY, LZ, CT>: tile TX x LY x LZ cells,
// CT coils per lane
enum { TG_2D_C1 = 0, TG_2D_C4 = 1, TG_2D_C8 = 2, TG_3D_C1 = 3, TG_3D_C8 = 4 };

static void tg_shape(int cfg, int t[3])
{
	static const int shapes[5][3] = { { 16, 32, 1 }, { 16, 16, 1 }, { 16, 8, 1 }, { 8, 8, 4 }, { 8, 4, 4 } };
	for (int a = 0; a < 3; a++)
		t[a] = shapes[cfg][a];
}

struct OpCtx {

	Geom g;
	int bin_edge = 0;	// gridding bin edge (0: default)
	int coils = 1;		// channels of the applies (picks the scatter's shape)
	const float4* traj;	// [M]
	const float* kb;
	float* ax = nullptr;	// [N0] roll-off along x
	float* ayz = nullptr;	// [N1*N2] roll-off along y,z with 1/sqrt(npix)
	Work w;
	Csr csr;		// set in deterministic mode
	Bins bins;		// binned gridding (all modes)
	const float2* wgt = nullptr;	// [M, wgt_c] weights (optional)
	long wgt_c = 1;
	float2* wbuf = nullptr;		// [M, C] weighted k-space for the adjoint
};

static void free_bins(Bins& b, cudaStream_t st)
{
	void* ptrs[] = { b.perm, b.traj, b.sub_bin, b.sub_first, b.sub_count, b.sub_start, b.bin_start, b.work_tile,
			b.work_chunk, b.work_start, b.multi, b.foot, b.kperm };

	for (void* q : ptrs)
		if (q)
			cudaFreeAsync(q, st);

	b = Bins{};
}

static void free_csr(Csr& c, cudaStream_t st)
{
	if (c.row_ptr) cudaFreeAsync(c.row_ptr, st);
	if (c.col) cudaFreeAsync(c.col, st);
	if (c.val) cudaFreeAsync(c.val, st);
	c = Csr{};
}

static GridGeom grid_geom(const Geom& g)
{
	GridGeom gg;

	for (int i = 0; i < 3; i++) {

		gg.N[i] = g.N[i];
		gg.G[i] = g.G[i];
	}

	gg.gsz = g.gsz;
	gg.hw = g.width / 2.f;
	gg.periodic = g.periodic;
	gg.chain = g.chain;
	gg.os = g.os;
	gg.wg = g.width;
	return gg;
}

static int alloc_work(Work& w, const Geom& g, long C, cudaStream_t st)
{
	if (w.cap >= C)
		return BNUFFT_OK;

	if (w.grid) cudaFreeAsync(w.grid, st);
	if (w.t1) cudaFreeAsync(w.t1, st);
	if (w.t2) cudaFreeAsync(w.t2, st);
	w = Work{};

	CUDA_TRY(cudaMallocAsync(&w.grid, sizeof(float2) * g.gsz * C, st));
	CUDA_TRY(cudaMallocAsync(&w.t1, sizeof(float2) * (long)g.G[0] * g.N[1] * g.N[2] * C, st));

	if (g.G[2] > 1)
		CUDA_TRY(cudaMallocAsync(&w.t2, sizeof(float2) * (long)g.G[0] * g.G[1] * g.N[2] * C, st));

	w.cap = C;
	return BNUFFT_OK;
}

static void free_work(Work& w, cudaStream_t st)
{
	if (w.grid) cudaFreeAsync(w.grid, st);
	if (w.t1) cudaFreeAsync(w.t1, st);
	if (w.t2) cudaFreeAsync(w.t2, st);
	w = Work{};
}

static int init_geom(Geom& g, const long dims3[3], long M, float os, float width, int periodic)
{
	g.nd = 0;
	g.npix = 1;
	g.gsz = 1;

	g.chain = (2.f != os);

	for (int i = 0; i < 3; i++) {

		g.N[i] = (int)dims3[i];
		// os != 2: the grid of lround(os N) cells of nufft_create_chain
		// (src/noncart/nufft_chain.c:205-208)
		g.G[i] = (dims3[i] > 1) ? (g.chain ? (int)std::lround((double)os * (double)dims3[i]) : (int)(2 * dims3[i])) : 1;

		if (dims3[i] > 1) {

			g.nd++;

			if (0 != dims3[i] % 2)
				return fail(BNUFFT_ERR_UNSUPPORTED, "odd image size %ld (even sizes are built)", dims3[i]);

			if (g.chain && ((0 != g.G[i] % 2) || (g.G[i] <= g.N[i])))
				return fail(BNUFFT_ERR_UNSUPPORTED, "oversampled grid of %d cells for %ld pixels (an even grid larger than the image is built)",
						g.G[i], dims3[i]);

			if (!supported_len(g.G[i]))
				return fail(BNUFFT_ERR_UNSUPPORTED, "grid length %d on axis %d", g.G[i], i);
		}

		g.npix *= g.N[i];
		g.gsz *= g.G[i];
	}

	if (dims3[0] <= 1)
		return fail(BNUFFT_ERR_ARG, "dim 0 must be transformed");

	if ((dims3[2] > 1) && (dims3[1] <= 1))
		return fail(BNUFFT_ERR_UNSUPPORTED, "3D with singleton y");

	g.M = M;
	g.os = os;
	g.width = width;
	g.periodic = periodic;
	return BNUFFT_OK;
}

// roll-off tables of a geometry, cached per device (computed once on the host)
struct RollKey {

	int n[3];
	float os, width;

	bool operator<(const RollKey& o) const
	{
		return std::memcmp(this, &o, sizeof *this) < 0;
	}
};

static std::map<std::pair<int, RollKey>, std::pair<float*, float*>> g_roll;

// separable roll-off of an N[0] x N[1] x N[2] image: ax[x] and
// ayz[y + N[1] z] (the latter with the unitary 1/sqrt(npix) folded in)
static void rolloff_host(const int N[3], float os, float width, float* ax, float* ayz)
{
	double beta = kernel_beta(os, width);
	double i0b = bessel_i0(beta);
	double sc = 1. / sqrt((double)N[0] * (double)N[1] * (double)N[2]);

	if (2.f != os) {	// the chain: unitary centred FFT on the lround(os N) grid, times os^(d/2)

		double gs = 1.;
		int nd = 0;

		for (int i = 0; i < 3; i++)
			if (N[i] > 1) {

				gs *= (double)std::lround((double)os * (double)N[i]);
				nd++;
			}

		sc = pow((double)os, 0.5 * nd) / sqrt(gs);
	}

	for (int x = 0; x < N[0]; x++)
		ax[x] = (float)rolloff_axis(N[0], x, os, width, beta, i0b);

	for (int z = 0; z < N[2]; z++)
		for (int y = 0; y < N[1]; y++)
			ayz[y + (size_t)N[1] * z] = (float)(rolloff_axis(N[1], y, os, width, beta, i0b)
						* rolloff_axis(N[2], z, os, width, beta, i0b) * sc);
}

static int init_rolloff(OpCtx& op, cudaStream_t st)
{
	const Geom& g = op.g;
	RollKey key;
	std::memset(&key, 0, sizeof key);

	for (int i = 0; i < 3; i++)
		key.n[i] = g.N[i];

	key.os = g.os;
	key.width = g.width;

	int dev;
	CUDA_TRY(cudaGetDevice(&dev));
	std::lock_guard<std::mutex> lock(g_tab_mutex);
	auto it = g_roll.find(std::make_pair(dev, key));

	if (it != g_roll.end()) {

		op.ax = it->second.first;
		op.ayz = it->second.second;
		return BNUFFT_OK;
	}

	std::vector<float> ax(g.N[0]);
	std::vector<float> ayz((size_t)g.N[1] * g.N[2]);
	rolloff_host(g.N, g.os, g.width, ax.data(), ayz.data());
	float* dax = nullptr;
	float* dayz = nullptr;
	CUDA_TRY(cudaMalloc(&dax, sizeof(float) * ax.size()));
	CUDA_TRY(cudaMalloc(&dayz, sizeof(float) * ayz.size()));
	CUDA_TRY(cudaMemcpy(dax, ax.data(), sizeof(float) * ax.size(), cudaMemcpyHostToDevice));
	CUDA_TRY(cudaMemcpy(dayz, ayz.data(), sizeof(float) * ayz.size(), cudaMemcpyHostToDevice));
	g_roll[std::make_pair(dev, key)] = std::make_pair(dax, dayz);
	op.ax = dax;
	op.ayz = dayz;
	(void)st;
	return BNUFFT_OK;
}

// column passes of the forward spectrum: row-transformed t1 -> grid
static int op_spectrum_cols(OpCtx& op, long C, float2* grid, cudaStream_t st)
{
	const Geom& g = op.g;

	if (1 == g.G[1]) {	// 1D: row pass is the whole transform

		CUDA_TRY(cudaMemcpyAsync(grid, op.w.t1, sizeof(float2) * g.gsz * C, cudaMemcpyDeviceToDevice, st));
		return BNUFFT_OK;
	}

	if (1 == g.G[2]) {

		return cols(g.G[1], 0, op.w.t1, g.G[0], (long)g.G[0] * g.N[1], g.N[1], 1,
				grid, g.G[0], (long)g.G[0] * g.G[1], g.G[1], 0, g.G[0], C, nullptr, 0, 1, 0, st);
	}

	TRY(cols(g.G[1], 0, op.w.t1, g.G[0], (long)g.G[0] * g.N[1], g.N[1], 1,
			op.w.t2, g.G[0], (long)g.G[0] * g.G[1], g.G[1], 0, g.G[0], (long)g.N[2] * C, nullptr, 0, 1, 0, st));

	long plane = (long)g.G[0] * g.G[1];

	return cols(g.G[2], 0, op.w.t2, plane, plane * g.N[2], g.N[2], 1,
			grid, plane, plane * g.G[2], g.G[2], 0, (int)plane, C, nullptr, 0, 1, 0, st);
}

// image [N0, N1*N2, C] (maps: image [N0, N1*N2] times maps [.., C]) -> grid
static int op_spectrum(OpCtx& op, const float2* img, const float2* maps, bool apod, long C, float2* grid, cudaStream_t st)
{
	const Geom& g = op.g;
	long YZ = (long)g.N[1] * g.N[2];

	TRY(rows_fwd(g.G[0], img, maps, apod ? op.ax : nullptr, op.ayz, g.N[0], YZ, YZ * C, op.w.t1, st));
	return op_spectrum_cols(op, C, grid, st);
}

// CG hooks of the final row pass: p for the partial p^H (partial sums)
struct DotHook {

	const float2* p = nullptr;
	double* part = nullptr;
	const int* done = nullptr;
	int* nblocks = nullptr;
};

// grid -> image (maps: sum over coils into `groups` partials of [N0, N1*N2])
static int op_spectrum_adjoint(OpCtx& op, const float2* grid, const float2* maps, bool apod, long C, int cpg,
		float2* out, cudaStream_t st, const DotHook& dh = DotHook())
{
	const Geom& g = op.g;
	long YZ = (long)g.N[1] * g.N[2];
	const float2* rows_in = grid;

	if (g.G[1] > 1) {

		if (1 == g.G[2]) {

			TRY(cols(g.G[1], 1, grid, g.G[0], (long)g.G[0] * g.G[1], g.G[1], 0,
					op.w.t1, g.G[0], (long)g.G[0] * g.N[1], g.N[1], 1, g.G[0], C, nullptr, 0, 1, 0, st));

		} else {

			long plane = (long)g.G[0] * g.G[1];

			TRY(cols(g.G[2], 1, grid, plane, plane * g.G[2], g.G[2], 0,
					op.w.t2, plane, plane * g.N[2], g.N[2], 1, (int)plane, C, nullptr, 0, 1, 0, st));
			TRY(cols(g.G[1], 1, op.w.t2, g.G[0], plane, g.G[1], 0,
					op.w.t1, g.G[0], (long)g.G[0] * g.N[1], g.N[1], 1, g.G[0], (long)g.N[2] * C, nullptr, 0, 1, 0, st));
		}

		rows_in = op.w.t1;
	}

	return rows_inv(g.G[0], rows_in, maps, apod ? op.ax : nullptr, op.ayz, g.N[0], YZ, (int)C, maps ? cpg : 1, out, st,
			dh.p, dh.part, dh.done, dh.nblocks);
}

static int degrid(OpCtx& op, const float2* grid, long C, float2* ksp, cudaStream_t st)
{
	if (op.bins.perm && (6.f == op.g.width)) {

		const Bins& b = op.bins;
		cudaEvent_t pe = prof_begin("degrid", st);
		unsigned nb = (unsigned)((op.g.M + BIN_THREADS - 1) / BIN_THREADS);

		if (op.g.G[2] > 1)
			k_degrid6<6><<<nb, BIN_THREADS, 0, st>>>(b.traj, b.perm, op.g.M, grid_geom(op.g), (int)C, grid, ksp, op.kb);
		else
			k_degrid6<1><<<nb, BIN_THREADS, 0, st>>>(b.traj, b.perm, op.g.M, grid_geom(op.g), (int)C, grid, ksp, op.kb);

		prof_end(pe, st);
		LAUNCHED();
		return BNUFFT_OK;
	}

	int cpc = (int)std::min<long>(C, 8);
	dim3 blocks((unsigned)((op.g.M + 127) / 128), (unsigned)((C + cpc - 1) / cpc));
	cudaEvent_t pe = prof_begin("degrid", st);
	k_degrid<<<blocks, 128, 0, st>>>(op.traj, op.g.M, grid_geom(op.g), (int)C, cpc, grid, ksp, op.kb);
	prof_end(pe, st);
	LAUNCHED();
	return BNUFFT_OK;
}

static int grid_adj(OpCtx& op, const float2* ksp, long C, float2* grid, cudaStream_t st)
{
	if (op.csr.row_ptr) {	// deterministic: fixed-order gather per cell

		int cpc = (int)std::min<long>(C, 8);
		dim3 blocks((unsigned)((op.g.gsz * 32 + 255) / 256), (unsigned)((C + cpc - 1) / cpc));
		cudaEvent_t pe = prof_begin("grid", st);
		k_grid_csr<<<blocks, 256, 0, st>>>(op.csr.row_ptr, op.csr.col, op.csr.val, op.g.gsz, op.g.M, (int)C, cpc, ksp, grid);
		prof_end(pe, st);
		LAUNCHED();
		return BNUFFT_OK;
	}

	if (op.bins.perm && (op.bins.tg_cfg >= 0)) {	// output-stationary tiles: no clearing pass

		Bins& b = op.bins;
		const GridGeom gg = grid_geom(op.g);
		TileWork tw = { b.bin_start, b.work_tile, b.work_chunk, b.work_start + b.ntiles, b.multi, b.foot, b.cand };
		int sorted = 0;

		// k-space in bin order (one pass), so the tiles read their samples'
		// values coalesced
		if (C > 1) {

			if (b.kperm_c < C) {	// more channels than the plan was made for (not while capturing)

				if (b.kperm)
					cudaFreeAsync(b.kperm, st);

				b.kperm = nullptr;
				b.kperm_c = 0;
				CUDA_TRY(cudaMallocAsync(&b.kperm, sizeof(float2) * op.g.M * C, st));
				b.kperm_c = C;
			}

			k_permute_ksp<<<vec_blocks(op.g.M * C, 256, 16 * 148), 256, 0, st>>>(b.kperm, ksp, b.perm, op.g.M, (int)C);
			LAUNCHED();
			ksp = b.kperm;
			sorted = 1;
		}

		cudaEvent_t pe = prof_begin("grid", st);
		k_zero_tiles<<<(unsigned)std::min<long>(b.ntiles, 8 * 148), 256, 0, st>>>(grid, gg, b.bg, b.multi, b.ntiles, (int)C);
		LAUNCHED();
		int t[3];
		tg_shape(b.tg_cfg, t);
		const int gpw = 32 / (t[1] * t[2]);
		const int ct = (TG_3D_C8 == b.tg_cfg) ? 4 : ((TG_2D_C8 == b.tg_cfg) || (TG_2D_C4 == b.tg_cfg) ? 2 : 1);
		const long ncq = (C + gpw * ct - 1) / (gpw * ct);
		const unsigned nblk = (unsigned)((b.nwork_max * ncq + TG_WARPS - 1) / TG_WARPS);

		switch (b.tg_cfg) {
		case TG_2D_C1:
			k_grid6_tiles<16, 32, 1, 1><<<nblk, 32 * TG_WARPS, 0, st>>>(b.perm, op.g.M, gg, b.bg, tw, (int)C, ksp, sorted, grid);
			break;
		case TG_2D_C4:
			k_grid6_tiles<16, 16, 1, 2><<<nblk, 32 * TG_WARPS, 0, st>>>(b.perm, op.g.M, gg, b.bg, tw, (int)C, ksp, sorted, grid);
			break;
		case TG_2D_C8:
			k_grid6_tiles<16, 8, 1, 2><<<nblk, 32 * TG_WARPS, 0, st>>>(b.perm, op.g.M, gg, b.bg, tw, (int)C, ksp, sorted, grid);
			break;
		case TG_3D_C1:
			k_grid6_tiles<8, 8, 4, 1><<<nblk, 32 * TG_WARPS, 0, st>>>(b.perm, op.g.M, gg, b.bg, tw, (int)C, ksp, sorted, grid);
			break;
		default:
			k_grid6_tiles<8, 4, 4, 4><<<nblk, 32 * TG_WARPS, 0, st>>>(b.perm, op.g.M, gg, b.bg, tw, (int)C, ksp, sorted, grid);
			break;
		}

		prof_end(pe, st);
		LAUNCHED();
		return BNUFFT_OK;
	}

	CUDA_TRY(cudaMemsetAsync(grid, 0, sizeof(float2) * op.g.gsz * C, st));

	if (op.bins.perm && (6.f == op.g.width) && (gridding_kind() >= 1)) {

		const Bins& b = op.bins;
		cudaEvent_t pe = prof_begin("grid", st);
		unsigned nb = (unsigned)((op.g.M + BIN_THREADS - 1) / BIN_THREADS);

		if (op.g.G[2] > 1)
			k_grid6_atomic<6><<<nb, BIN_THREADS, 0, st>>>(b.traj, b.perm, op.g.M, grid_geom(op.g), (int)C, ksp, grid, op.kb);
		else
			k_grid6_atomic<1><<<nb, BIN_THREADS, 0, st>>>(b.traj, b.perm, op.g.M, grid_geom(op.g), (int)C, ksp, grid, op.kb);

		prof_end(pe, st);
		LAUNCHED();
		return BNUFFT_OK;
	}

	if (op.bins.perm && (6.f == op.g.width)) {

		const Bins& b = op.bins;
		int cc = (int)std::min<long>(b.cc, C);
		size_t smem = sizeof(float2) * b.bg.ncells * cc;
		cudaEvent_t pe = prof_begin("grid", st);

		if (op.g.G[2] > 1) {

			TRY(prep_kernel(k_grid6_binned<6>, smem));
			k_grid6_binned<6><<<b.nsub, BIN_THREADS, smem, st>>>(b.traj, b.perm, op.g.M, grid_geom(op.g), b.bg,
					b.sub_bin, b.sub_first, b.sub_count, b.nsub_dev, (int)C, cc, ksp, grid, op.kb);

		} else {

			TRY(prep_kernel(k_grid6_binned<1>, smem));
			k_grid6_binned<1><<<b.nsub, BIN_THREADS, smem, st>>>(b.traj, b.perm, op.g.M, grid_geom(op.g), b.bg,
					b.sub_bin, b.sub_first, b.sub_count, b.nsub_dev, (int)C, cc, ksp, grid, op.kb);
		}

		prof_end(pe, st);
		LAUNCHED();
		return BNUFFT_OK;
	}

	int cpc = (int)std::min<long>(C, 8);
	dim3 blocks((unsigned)((op.g.M + 127) / 128), (unsigned)((C + cpc - 1) / cpc));
	cudaEvent_t pe = prof_begin("grid", st);
	k_grid_atomic<<<blocks, 128, 0, st>>>(op.traj, op.g.M, grid_geom(op.g), (int)C, cpc, ksp, grid, op.kb);
	prof_end(pe, st);
	LAUNCHED();
	return BNUFFT_OK;
}

// Build the CSR interpolation matrix of op's trajectory (stable sort by
// cell * M + sample, so each row lists its samples in increasing order).
static int build_csr(OpCtx& op, cudaStream_t st)
{
	const Geom& g = op.g;
	int slots_z = (g.G[2] > 1) ? CSR_TAPS_AXIS : 1;
	long slots = (long)CSR_TAPS_AXIS * CSR_TAPS_AXIS * slots_z;
	long n = g.M * slots;

	if ((g.M >= (1L << 31)) || ((unsigned long long)g.gsz * (unsigned long long)g.M >= (~0ull >> 1)) || (n >= (1L << 31)))
		return fail(BNUFFT_ERR_UNSUPPORTED, "deterministic gridding: %ld samples x %ld cells is too large", g.M, g.gsz);

	unsigned long long *keys = nullptr, *keys2 = nullptr;
	float *vals = nullptr, *vals2 = nullptr;
	int* counts = nullptr;
	void* tmp = nullptr;
	size_t tmp_bytes = 0;
	CUDA_TRY(cudaMallocAsync(&keys, sizeof(unsigned long long) * n, st));
	CUDA_TRY(cudaMallocAsync(&keys2, sizeof(unsigned long long) * n, st));
	CUDA_TRY(cudaMallocAsync(&vals, sizeof(float) * n, st));
	CUDA_TRY(cudaMallocAsync(&vals2, sizeof(float) * n, st));

	k_csr_keys<<<(unsigned)((g.M + 127) / 128), 128, 0, st>>>(op.traj, g.M, grid_geom(g), op.kb, keys, vals, slots_z);
	LAUNCHED();

	CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys2, vals, vals2, (int)n, 0, 64, st));
	CUDA_TRY(cudaMallocAsync(&tmp, tmp_bytes, st));
	CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, vals, vals2, (int)n, 0, 64, st));
	g_launches.fetch_add(1, std::memory_order_relaxed);

	// entries with a valid key come first; count them per cell
	Csr& c = op.csr;
	CUDA_TRY(cudaMallocAsync(&counts, sizeof(int) * (g.gsz + 1), st));
	CUDA_TRY(cudaMemsetAsync(counts, 0, sizeof(int) * (g.gsz + 1), st));
	CUDA_TRY(cudaMallocAsync(&c.row_ptr, sizeof(long) * (g.gsz + 1), st));

	// number of valid entries: taps of every sample (host needs it for sizes)
	int* col_all = nullptr;
	CUDA_TRY(cudaMallocAsync(&col_all, sizeof(int) * n, st));
	k_csr_fill_valid<<<vec_blocks(n), RED_THREADS, 0, st>>>(keys2, n, g.M, g.gsz, col_all, counts);
	LAUNCHED();

	size_t scan_bytes = 0;
	void* scan_tmp = nullptr;
	CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, counts, c.row_ptr, (int)(g.gsz + 1), st));
	CUDA_TRY(cudaMallocAsync(&scan_tmp, scan_bytes, st));
	CUDA_TRY(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, counts, c.row_ptr, (int)(g.gsz + 1), st));
	g_launches.fetch_add(1, std::memory_order_relaxed);

	long nnz = 0;
	CUDA_TRY(cudaMemcpyAsync(&nnz, c.row_ptr + g.gsz, sizeof(long), cudaMemcpyDeviceToHost, st));
	CUDA_TRY(cudaStreamSynchronize(st));
	c.nnz = nnz;

	// valid entries are the first nnz of the sorted arrays
	c.col = col_all;
	c.val = vals2;

	cudaFreeAsync(keys, st);
	cudaFreeAsync(keys2, st);
	cudaFreeAsync(vals, st);
	cudaFreeAsync(counts, st);
	cudaFreeAsync(tmp, st);
	cudaFreeAsync(scan_tmp, st);
	return BNUFFT_OK;
}

// Sort the samples by bin and cut bins into sub-blocks (plan time).
static int build_bins(OpCtx& op, cudaStream_t st)
{
	const Geom& g = op.g;
	Bins& b = op.bins;
	BinGeom& bg = b.bg;
	const int bs_axis = op.bin_edge ? op.bin_edge : ((g.G[2] > 1) ? 16 : 32);
	long nbins = 1;
	bg.ncells = 1;

	// the output-stationary scatter (default for width 6 unless a bin edge
	// is set): bins are its tiles; it needs three bins per transformed axis
	// and, on periodic grids, room for an unambiguous footprint offset
	b.tg_cfg = -1;

	// measured on B200: it wins for multi-channel problems (8-coil 128^3
	// kooshball: 10.5 against 28.2 ms; 16-coil 256^2 radial: 122 against
	// 144 us), while single-channel problems (little work per candidate
	// sample) are faster with the global-atomic scatter (256^2, 402 spokes:
	// 55 against 122 us); BNUFFT_GRIDDING=lines selects it everywhere
	const bool tg_want = (2 == gridding_kind()) ? (op.coils >= 2) : (3 == gridding_kind());

	if ((6.f == g.width) && (0 == op.bin_edge) && tg_want && (g.G[0] > 1) && (g.G[1] > 1)) {

		const bool d3 = (g.G[2] > 1);
		int cfg = d3 ? ((op.coils >= 2) ? TG_3D_C8 : TG_3D_C1)
				: ((op.coils >= 5) ? TG_2D_C8 : ((op.coils >= 2) ? TG_2D_C4 : TG_2D_C1));
		int t[3];
		tg_shape(cfg, t);
		bool ok = true;

		for (int a = 0; a < 3; a++)
			if (g.G[a] > 1)
				ok = ok && (g.G[a] >= 3 * t[a]) && (!g.periodic || (g.G[a] > 2 * t[a] + 16));

		if (ok)
			b.tg_cfg = cfg;
	}

	for (int a = 0; a < 3; a++) {

		int t[3] = { bs_axis, bs_axis, bs_axis };

		if (b.tg_cfg >= 0)
			tg_shape(b.tg_cfg, t);

		bg.bs[a] = (g.G[a] > 1) ? std::min(t[a], g.G[a]) : 1;
		bg.nb[a] = (g.G[a] + bg.bs[a] - 1) / bg.bs[a];
		bg.tile[a] = (g.G[a] > 1) ? bg.bs[a] + 2 * BIN_HALO : 1;
		nbins *= bg.nb[a];
		bg.ncells *= bg.tile[a];
	}

	if ((g.M >= (1L << 31)) || (nbins >= (1L << 31)))
		return fail(BNUFFT_ERR_UNSUPPORTED, "binning: %ld samples, %ld bins", g.M, nbins);

	unsigned *keys = nullptr, *keys2 = nullptr;
	int *vals = nullptr, *counts = nullptr, *bin_start = nullptr, *nsub = nullptr, *sub_start = nullptr;
	void* tmp = nullptr;
	size_t tmp_bytes = 0, tmp2 = 0;
	long M = g.M;

	CUDA_TRY(cudaMallocAsync(&keys, sizeof(unsigned) * M, st));
	CUDA_TRY(cudaMallocAsync(&keys2, sizeof(unsigned) * M, st));
	CUDA_TRY(cudaMallocAsync(&vals, sizeof(int) * M, st));
	CUDA_TRY(cudaMallocAsync(&b.perm, sizeof(int) * M, st));
	CUDA_TRY(cudaMallocAsync(&b.traj, sizeof(float4) * M, st));
	CUDA_TRY(cudaMallocAsync(&counts, sizeof(int) * (nbins + 1), st));
	CUDA_TRY(cudaMallocAsync(&bin_start, sizeof(int) * (nbins + 1), st));
	CUDA_TRY(cudaMallocAsync(&nsub, sizeof(int) * (nbins + 1), st));
	CUDA_TRY(cudaMallocAsync(&sub_start, sizeof(int) * (nbins + 1), st));
	CUDA_TRY(cudaMemsetAsync(counts, 0, sizeof(int) * (nbins + 1), st));

	k_bin_keys<<<vec_blocks(M), RED_THREADS, 0, st>>>(op.traj, M, grid_geom(g), bg, keys, vals, counts);
	LAUNCHED();

	int end_bit = 1;

	while ((1L << end_bit) < nbins)
		end_bit++;

	CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys2, vals, b.perm, (int)M, 0, end_bit, st));
	CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp2, counts, bin_start, (int)(nbins + 1), st));
	tmp_bytes = std::max(tmp_bytes, tmp2);
	CUDA_TRY(cudaMallocAsync(&tmp, tmp_bytes, st));
	CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, vals, b.perm, (int)M, 0, end_bit, st));
	CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, counts, bin_start, (int)(nbins + 1), st));
	g_launches.fetch_add(2, std::memory_order_relaxed);

	// sub-blocks per bin: ceil(count / sub); their start indices. A
	// sub-block is one block of the tile scatter, which clears and flushes
	// its tile once: large sub-blocks amortise that, small ones balance the
	// dense bins at the k-space centre
	int sub = BIN_SUB;

	if (const char* e = getenv("BNUFFT_GRID_SUB"))
		sub = std::max(64, std::min(1 << 20, atoi(e)));

	k_bin_nsub<<<vec_blocks(nbins + 1), RED_THREADS, 0, st>>>(bin_start, (int)nbins, sub, nsub);
	LAUNCHED();
	CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, nsub, sub_start, (int)(nbins + 1), st));
	g_launches.fetch_add(1, std::memory_order_relaxed);

	// the number of sub-blocks stays on the device (no host round trip);
	// launches use the upper bound nbins + M / BIN_SUB and surplus blocks exit
	long total = nbins + M / sub + 1;
	b.nsub = (int)total;
	b.sub_start = sub_start;
	b.nsub_dev = sub_start + nbins;

	CUDA_TRY(cudaMallocAsync(&b.sub_bin, sizeof(int) * total, st));
	CUDA_TRY(cudaMallocAsync(&b.sub_first, sizeof(int) * total, st));
	CUDA_TRY(cudaMallocAsync(&b.sub_count, sizeof(int) * total, st));
	k_sub_fill<<<vec_blocks(nbins), RED_THREADS, 0, st>>>(bin_start, sub_start, (int)nbins, sub, b.sub_bin, b.sub_first, b.sub_count);
	LAUNCHED();
	k_gather_traj<<<vec_blocks(M), RED_THREADS, 0, st>>>(b.traj, op.traj, b.perm, M);
	LAUNCHED();

	// coil tiles per pass: as many as fit in ~110 KB of shared memory
	b.cc = (int)std::max(1L, std::min(8L, (110L * 1024) / (long)(sizeof(float2) * bg.ncells)));

	// work items of the output-stationary scatter: each tile's candidates
	// (the samples of its neighbour bins) in chunks of b.cand
	if (b.tg_cfg >= 0) {

		const long nt = nbins;
		const int nneigh = (g.G[2] > 1) ? 27 : 9;
		int* nwork = nullptr;
		void* wtmp = nullptr;
		size_t wtmp_bytes = 0;
		b.ntiles = nt;
		b.bin_start = bin_start;
		bin_start = nullptr;	// kept by the plan
		b.cand = (g.G[2] > 1) ? 1024 : 256;	// measured best (256..1024 tried)

		if (const char* e = getenv("BNUFFT_GRID_CAND"))	// tuning knob: candidates per work item
			b.cand = std::max(64, std::min(4096, atoi(e)));

		b.nwork_max = nt + (M * nneigh + b.cand - 1) / b.cand;

		if (b.nwork_max >= (1L << 31))
			return fail(BNUFFT_ERR_UNSUPPORTED, "gridding: %ld work items", b.nwork_max);

		CUDA_TRY(cudaMallocAsync(&nwork, sizeof(int) * (nt + 1), st));
		CUDA_TRY(cudaMallocAsync(&b.work_start, sizeof(int) * (nt + 1), st));
		CUDA_TRY(cudaMallocAsync(&b.multi, nt, st));
		CUDA_TRY(cudaMallocAsync(&b.work_tile, sizeof(int) * b.nwork_max, st));
		CUDA_TRY(cudaMallocAsync(&b.work_chunk, sizeof(int) * b.nwork_max, st));
		CUDA_TRY(cudaMemsetAsync(nwork + nt, 0, sizeof(int), st));
		k_tile_cand<<<vec_blocks(nt), RED_THREADS, 0, st>>>(b.bin_start, bg, g.periodic, nt, b.cand, nwork, b.multi);
		LAUNCHED();
		CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, wtmp_bytes, nwork, b.work_start, (int)(nt + 1), st));
		CUDA_TRY(cudaMallocAsync(&wtmp, wtmp_bytes, st));
		CUDA_TRY(cub::DeviceScan::ExclusiveSum(wtmp, wtmp_bytes, nwork, b.work_start, (int)(nt + 1), st));
		g_launches.fetch_add(1, std::memory_order_relaxed);
		k_work_fill<<<vec_blocks(nt), RED_THREADS, 0, st>>>(b.work_start, nt, b.work_tile, b.work_chunk);
		LAUNCHED();
		cudaFreeAsync(nwork, st);
		cudaFreeAsync(wtmp, st);

		// the samples' footprints (start cells and weights): they depend on
		// the trajectory only, so every apply reads them instead of
		// recomputing 18 table lookups per sample and tile
		CUDA_TRY(cudaMallocAsync(&b.foot, sizeof(float4) * FOOT_F4 * M, st));
		k_foot<<<vec_blocks(M, 128, 8 * 148), 128, 0, st>>>(b.traj, M, grid_geom(g), op.kb, b.foot);
		LAUNCHED();

		// the bin-ordered k-space of the applies, allocated here so that
		// applies allocate nothing (their solves can then be captured into
		// graphs and nested as child graphs)
		if (op.coils > 1) {

			CUDA_TRY(cudaMallocAsync(&b.kperm, sizeof(float2) * M * op.coils, st));
			b.kperm_c = op.coils;
		}
	}

	void* frees[] = { keys, keys2, vals, counts, bin_start, nsub, tmp };

	for (void* q : frees)
		if (q)
			cudaFreeAsync(q, st);

	return BNUFFT_OK;
}

// forward NUFFT: cim [npix, C] -> ksp [M, C] (maps: single image times maps)
static int op_forward(OpCtx& op, const float2* cim, const float2* maps, long C, float2* ksp, cudaStream_t st)
{
	TRY(alloc_work(op.w, op.g, C, st));
	TRY(op_spectrum(op, cim, maps, true, C, op.w.grid, st));
	TRY(degrid(op, op.w.grid, C, ksp, st));

	if (op.wgt) {

		k_weight<<<vec_blocks(op.g.M * C), RED_THREADS, 0, st>>>(ksp, ksp, op.wgt, op.g.M, C, op.wgt_c, 0);
		LAUNCHED();
	}

	return BNUFFT_OK;
}

// adjoint NUFFT: ksp [M, C] -> cim [npix, C] (maps: partial coil sums)
static int op_adjoint(OpCtx& op, const float2* ksp, const float2* maps, long C, int cpg, float2* out, cudaStream_t st,
		const DotHook& dh = DotHook())
{
	TRY(alloc_work(op.w, op.g, C, st));

	if (op.wgt) {

		if (!op.wbuf)
			CUDA_TRY(cudaMallocAsync(&op.wbuf, sizeof(float2) * op.g.M * C, st));

		k_weight<<<vec_blocks(op.g.M * C), RED_THREADS, 0, st>>>(op.wbuf, ksp, op.wgt, op.g.M, C, op.wgt_c, 1);
		LAUNCHED();
		ksp = op.wbuf;
	}

	TRY(grid_adj(op, ksp, C, op.w.grid, st));
	return op_spectrum_adjoint(op, op.w.grid, maps, true, C, cpg, out, st, dh);
}

// column passes of the Toeplitz product on the row-transformed t1 (in place)
static int op_toeplitz_cols(OpCtx& op, const float2* psf, long C, cudaStream_t st, const int* done = nullptr)
{
	const Geom& g = op.g;

	if (1 == g.G[1])
		return fail(BNUFFT_ERR_UNSUPPORTED, "Toeplitz normal for 1D");

	if (1 == g.G[2])
		return cols(g.G[1], 2, op.w.t1, g.G[0], (long)g.G[0] * g.N[1], g.N[1], 1,
				op.w.t1, g.G[0], (long)g.G[0] * g.N[1], g.N[1], 1, g.G[0], C, psf, g.G[0], 1, 0, st, done);

	long plane = (long)g.G[0] * g.G[1];

	TRY(cols(g.G[1], 0, op.w.t1, g.G[0], (long)g.G[0] * g.N[1], g.N[1], 1,
			op.w.t2, g.G[0], plane, g.G[1], 0, g.G[0], (long)g.N[2] * C, nullptr, 0, 1, 0, st, done));
	TRY(cols(g.G[2], 2, op.w.t2, plane, plane * g.N[2], g.N[2], 1,
			op.w.t2, plane, plane * g.N[2], g.N[2], 1, (int)plane, C, psf, plane, 1, 0, st, done));
	return cols(g.G[1], 1, op.w.t2, g.G[0], plane, g.G[1], 0,
			op.w.t1, g.G[0], (long)g.G[0] * g.N[1], g.N[1], 1, g.G[0], (long)g.N[2] * C, nullptr, 0, 1, 0, st, done);
}

// Toeplitz normal: E^H (psf . E x) per coil (maps: partial coil sums)
static int op_toeplitz(OpCtx& op, const float2* psf, const float2* x, const float2* maps, long C, int cpg,
		float2* out, cudaStream_t st)
{
	const Geom& g = op.g;
	long YZ = (long)g.N[1] * g.N[2];
	TRY(alloc_work(op.w, g, C, st));
	TRY(rows_fwd(g.G[0], x, maps, nullptr, nullptr, g.N[0], YZ, YZ * C, op.w.t1, st));
	TRY(op_toeplitz_cols(op, psf, C, st));
	return rows_inv(g.G[0], op.w.t1, maps, nullptr, nullptr, g.N[0], YZ, (int)C, maps ? cpg : 1, out, st);
}

// Toeplitz normal with a subspace basis (toeplitz_mult with the block PSF,
// src/noncart/nufft.c:1546-1625): the full 2N spectra of all Cc K channels,
// per cell and coil the K x K product with the block PSF (k_basis_mix), and
// back; the same unnormalised transforms as the single-PSF column pass.
static int op_toeplitz_basis(OpCtx& op, const float2* psfb, const float2* x, long Cc, int K, float2* out,
		cudaStream_t st)
{
	const Geom& g = op.g;
	const long C = Cc * K;
	long YZ = (long)g.N[1] * g.N[2];
	TRY(alloc_work(op.w, g, C, st));
	TRY(rows_fwd(g.G[0], x, nullptr, nullptr, nullptr, g.N[0], YZ, YZ * C, op.w.t1, st));
	float2* spec = op.w.grid;

	if (1 == g.G[2]) {

		TRY(cols(g.G[1], 0, op.w.t1, g.G[0], (long)g.G[0] * g.N[1], g.N[1], 1,
				spec, g.G[0], g.gsz, g.G[1], 0, g.G[0], C, nullptr, 0, 1, 0, st));
		k_basis_mix<<<vec_blocks(g.gsz * Cc), RED_THREADS, 0, st>>>(spec, psfb, g.gsz, Cc, K);
		LAUNCHED();
		TRY(cols(g.G[1], 1, spec, g.G[0], g.gsz, g.G[1], 0,
				op.w.t1, g.G[0], (long)g.G[0] * g.N[1], g.N[1], 1, g.G[0], C, nullptr, 0, 1, 0, st));

	} else {

		long plane = (long)g.G[0] * g.G[1];
		TRY(cols(g.G[1], 0, op.w.t1, g.G[0], (long)g.G[0] * g.N[1], g.N[1], 1,
				op.w.t2, g.G[0], plane, g.G[1], 0, g.G[0], (long)g.N[2] * C, nullptr, 0, 1, 0, st));
		TRY(cols(g.G[2], 0, op.w.t2, plane, plane * g.N[2], g.N[2], 1,
				spec, plane, g.gsz, g.G[2], 0, (int)plane, C, nullptr, 0, 1, 0, st));
		k_basis_mix<<<vec_blocks(g.gsz * Cc), RED_THREADS, 0, st>>>(spec, psfb, g.gsz, Cc, K);
		LAUNCHED();
		TRY(cols(g.G[2], 1, spec, plane, g.gsz, g.G[2], 0,
				op.w.t2, plane, plane * g.N[2], g.N[2], 1, (int)plane, C, nullptr, 0, 1, 0, st));
		TRY(cols(g.G[1], 1, op.w.t2, g.G[0], plane, g.G[1], 0,
				op.w.t1, g.G[0], (long)g.G[0] * g.N[1], g.N[1], 1, g.G[0], (long)g.N[2] * C, nullptr, 0, 1, 0, st));
	}

	return rows_inv(g.G[0], op.w.t1, nullptr, nullptr, nullptr, g.N[0], YZ, (int)C, 1, out, st);
}

// PSF on the 2N grid in DFT order, scaled by 1/npix so that the Toeplitz
// product needs no further normalisation (compute_psf2, src/noncart/nufft.c:727-776):
// psft = adjoint NUFFT of ones with trajectory 2*traj onto the 2N image,
// periodic gridding; psf = fftuc(psft) / npix.
// With a subspace basis (K coefficients over T frames of MrMs samples) the
// "ones" are the K^2 channels conj(B[t, k]) B[t, k'] |w|^2 and the result is
// the block PSF [K^2][gsz], pair k + K k' (compute_square_basis,
// src/noncart/nufft.c:470-505).
static int compute_psf(const Geom& g, const float2* traj_c, const float* kb, float2** psf_out, cudaStream_t st,
		bool deterministic, const float2* wgt, int bin_edge, const float2* basis = nullptr, int K = 1, int T = 1,
		long MrMs = 0)
{
	OpCtx in;
	in.bin_edge = bin_edge;
	long d2[3] = { g.G[0], g.G[1], g.G[2] };
	TRY(init_geom(in.g, d2, g.M, g.os, g.width, 1));
	const long nch = basis ? (long)K * K : 1;

	float4* t2 = nullptr;
	float2* ones = nullptr;
	float2* psft = nullptr;
	float2* psf = nullptr;
	CUDA_TRY(cudaMallocAsync(&t2, sizeof(float4) * g.M, st));
	CUDA_TRY(cudaMallocAsync(&ones, sizeof(float2) * g.M * nch, st));
	CUDA_TRY(cudaMallocAsync(&psft, sizeof(float2) * in.g.npix * nch, st));
	CUDA_TRY(cudaMallocAsync(&psf, sizeof(float2) * g.gsz * nch, st));

	k_traj_convert<<<vec_blocks(g.M), RED_THREADS, 0, st>>>(t2, traj_c, g.M, 2.f);
	LAUNCHED();
	if (basis)
		k_basis_psf_weights<<<vec_blocks(g.M * nch), RED_THREADS, 0, st>>>(ones, basis, wgt, MrMs, T, K);
	else if (wgt)	// compute_square_weights (src/noncart/nufft.c:509-518)
		k_weight_sq<<<vec_blocks(g.M), RED_THREADS, 0, st>>>(ones, wgt, g.M);
	else
		k_fill<<<vec_blocks(g.M), RED_THREADS, 0, st>>>(ones, g.M, make_float2(1.f, 0.f));

	LAUNCHED();

	in.traj = t2;
	in.kb = kb;
	TRY(init_rolloff(in, st));

	TRY(build_bins(in, st));

	if (deterministic)
		TRY(build_csr(in, st));

	TRY(op_adjoint(in, ones, nullptr, nch, 1, psft, st));
	free_csr(in.csr, st);
	free_bins(in.bins, st);

	// full 2N-point transform of the 2N image: input centred (ifftshift), output in DFT order
	OpCtx full;
	full.g = g;
	full.traj = nullptr;
	full.kb = kb;

	for (int i = 0; i < 3; i++)
		full.g.N[i] = g.G[i];	// input length L on every axis

	full.g.npix = g.gsz;
	TRY(alloc_work(full.w, full.g, nch, st));

	long YZ = (long)g.G[1] * g.G[2];
	TRY(rows_fwd(g.G[0], psft, nullptr, nullptr, nullptr, g.G[0], YZ, YZ * nch, full.w.t1, st));

	if (1 == g.G[2]) {

		TRY(cols(g.G[1], 0, full.w.t1, g.G[0], (long)g.G[0] * g.G[1], g.G[1], 1,
				psf, g.G[0], (long)g.G[0] * g.G[1], g.G[1], 0, g.G[0], nch, nullptr, 0, 1, 0, st));

	} else {

		long plane = (long)g.G[0] * g.G[1];

		TRY(cols(g.G[1], 0, full.w.t1, g.G[0], plane, g.G[1], 1,
				full.w.t2, g.G[0], plane, g.G[1], 0, g.G[0], (long)g.G[2] * nch, nullptr, 0, 1, 0, st));
		TRY(cols(g.G[2], 0, full.w.t2, plane, plane * g.G[2], g.G[2], 1,
				psf, plane, plane * g.G[2], g.G[2], 0, (int)plane, nch, nullptr, 0, 1, 0, st));
	}

	double sc = 1. / sqrt((double)g.gsz) / (double)g.npix;
	k_scale<<<vec_blocks(g.gsz * nch), RED_THREADS, 0, st>>>(psf, psf, g.gsz * nch, (float)sc);
	LAUNCHED();

	free_work(full.w, st);
	free_work(in.w, st);
	cudaFreeAsync(t2, st);
	cudaFreeAsync(ones, st);
	cudaFreeAsync(psft, st);

	*psf_out = psf;
	return BNUFFT_OK;
}

// ----------------------------------------------------------------------------
// dims helpers
// ----------------------------------------------------------------------------

static long prod(int n, const long* d)
{
	long p = 1;

	for (int i = 0; i < n; i++)
		p *= d[i];

	return p;
}

static bool on_device(const void* p)
{
	cudaPointerAttributes a;

	if (cudaSuccess != cudaPointerGetAttributes(&a, p)) {

		cudaGetLastError();
		return false;
	}

	return (cudaMemoryTypeDevice == a.type) || (cudaMemoryTypeManaged == a.type);
}

// per thread and device: an auxiliary compute stream with a fork / join
// event pair, and a copy stream with its event
struct AuxStream {

	cudaStream_t st = nullptr;
	cudaEvent_t fork = nullptr, join = nullptr;
	cudaStream_t cp = nullptr;
	cudaEvent_t copied = nullptr;
};

static const AuxStream* aux_stream(int dev)
{
	static thread_local std::map<int, AuxStream> aux;
	auto it = aux.find(dev);

	if (it != aux.end())
		return &it->second;

	AuxStream a;

	if ((cudaSuccess != cudaStreamCreateWithFlags(&a.st, cudaStreamNonBlocking))
	    || (cudaSuccess != cudaEventCreateWithFlags(&a.fork, cudaEventDisableTiming))
	    || (cudaSuccess != cudaEventCreateWithFlags(&a.join, cudaEventDisableTiming))
	    || (cudaSuccess != cudaStreamCreateWithFlags(&a.cp, cudaStreamNonBlocking))
	    || (cudaSuccess != cudaEventCreateWithFlags(&a.copied, cudaEventDisableTiming))) {

		cudaGetLastError();
		return nullptr;
	}

	// the library allocates and frees stream-ordered per model: keep the
	// device's default pool from returning its memory at every host
	// synchronisation (it would map it again for the next model)
	cudaMemPool_t pool;

	if (cudaSuccess == cudaDeviceGetDefaultMemPool(&pool, dev)) {

		uint64_t keep = UINT64_MAX;
		cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
	}

	cudaGetLastError();
	return &(aux[dev] = a);
}

// the copy stream of this thread and device (nullptr: none)
static cudaStream_t copy_stream()
{
	int dev = 0;

	if (cudaSuccess != cudaGetDevice(&dev))
		return nullptr;

	const AuxStream* aux = aux_stream(dev);
	return aux ? aux->cp : nullptr;
}

// host-to-device copy of a host array on the copy stream: st waits for it,
// and the call returns once the copy has read the host array (not after
// earlier work queued on st). dst must be allocated in the copy stream's
// order (copy_stream()), so that a block still in use by earlier work on
// st is never handed out for it.
static int copy_in(void* dst, const void* src, size_t bytes, cudaStream_t st)
{
	int dev = 0;
	CUDA_TRY(cudaGetDevice(&dev));
	const AuxStream* aux = aux_stream(dev);

	if (!aux) {

		CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
		CUDA_TRY(cudaStreamSynchronize(st));
		return BNUFFT_OK;
	}

	CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, aux->cp));
	CUDA_TRY(cudaEventRecord(aux->copied, aux->cp));
	CUDA_TRY(cudaStreamWaitEvent(st, aux->copied, 0));
	CUDA_TRY(cudaEventSynchronize(aux->copied));
	return BNUFFT_OK;
}

// staging of host data through device buffers (the e2e path)
// Staging buffers come from the stream-ordered pool (cudaMallocAsync) and go
// back to it in stream order, so host-pointer calls neither synchronise the
// device nor pay cudaMalloc. Host inputs are read asynchronously from pinned
// memory: keep them unchanged until the stream has caught up (as with
// cudaMemcpyAsync); calls with host outputs synchronise before returning.
struct Staged {

	void* dev = nullptr;
	bool owned = false;
	cudaStream_t st = nullptr;

	~Staged() { if (owned && dev) cudaFreeAsync(dev, st); }
};

static int stage_in(Staged& s, const void* p, size_t bytes, cudaStream_t st)
{
	if (on_device(p)) {

		s.dev = (void*)p;
		return BNUFFT_OK;
	}

	cudaStream_t cs = copy_stream();
	CUDA_TRY(cudaMallocAsync(&s.dev, bytes, cs ? cs : st));
	s.owned = true;
	s.st = st;
	return copy_in(s.dev, p, bytes, st);
}

static int stage_out_alloc(Staged& s, void* p, size_t bytes, cudaStream_t st = nullptr)
{
	if (on_device(p)) {

		s.dev = p;
		return BNUFFT_OK;
	}

	CUDA_TRY(cudaMallocAsync(&s.dev, bytes, st));
	s.owned = true;
	s.st = st;
	return BNUFFT_OK;
}

static int stage_out_copy(Staged& s, void* p, size_t bytes, cudaStream_t st)
{
	if (!s.owned)
		return BNUFFT_OK;

	CUDA_TRY(cudaMemcpyAsync(p, s.dev, bytes, cudaMemcpyDeviceToHost, st));
	CUDA_TRY(cudaStreamSynchronize(st));
	return BNUFFT_OK;
}

// ----------------------------------------------------------------------------
// NUFFT plan (C ABI)
// ----------------------------------------------------------------------------

struct bnufft_plan_s {

	int N;
	std::vector<long> ksp_dims, cim_dims, trj_dims;
	bnufft_conf conf;
	long C;			// batch (product of cim dims >= 3)
	OpCtx op;
	float4* traj = nullptr;
	float2* psf = nullptr;	// DFT order, includes 1/npix ([K^2][gsz] with a basis)
	float2* wgt = nullptr;	// weights copy [M, wgt_c]
	// subspace basis: K = nb coefficients over T frames of MrMs samples each
	// (nb = 0 without one); the op's samples are all frames' (M = MrMs T),
	// its channels (coil c, coefficient k) at c + Cc k
	int nb = 0;
	int T = 1;
	long Cc = 1;
	long MrMs = 0;
	float2* basis = nullptr;	// [T, K], element t + T k
	float2* pinv = nullptr;	// circulant preconditioner 1/pre, [N0, N1*N2] DFT order (on demand)
	// Toeplitz normal on a power-of-two circulant embedding when 2N is not a
	// power of two: geometry with G = E >= 2N and the PSF re-embedded there
	bool embed = false;
	OpCtx toe;
	float2* psf_t = nullptr;
	cudaStream_t st0;
	// the PSF chain (and a pics model's preconditioner spectrum) runs on the
	// auxiliary stream; this event is recorded after it
	cudaEvent_t psf_ev = nullptr;
};

// A stream about to use the PSF, its embedding or the preconditioner
// spectrum first waits for the auxiliary stream's work that builds them, so
// the model's other set-up and the solve's adjoint run meanwhile. Skipped
// while the stream captures a graph (captures of whole solves are preceded
// by a host wait for that work; the CG loop graph is launched after a wait).
static void psf_wait(const bnufft_plan_s* p, cudaStream_t st)
{
	if (!p->psf_ev)
		return;

	cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;

	if (cudaSuccess != cudaStreamIsCapturing(st, &cs)) {

		cudaGetLastError();
		return;
	}

	if (cudaStreamCaptureStatusNone == cs)
		cudaStreamWaitEvent(st, p->psf_ev, 0);
}

static OpCtx& toe_ctx(bnufft_plan_s* p) { return p->embed ? p->toe : p->op; }

static const float2* toe_psf(const bnufft_plan_s* p, cudaStream_t st)
{
	psf_wait(p, st);
	return p->embed ? p->psf_t : p->psf;
}

static const float2* precond_spec(const bnufft_plan_s* p, cudaStream_t st)
{
	psf_wait(p, st);
	return p->pinv;
}

// q'[i] = scale * q[d mod L] at d = i (i < N) or i - E (i > E - N), else 0,
// per axis: the kernel of the Toeplitz operator (|d| < N) moved from the
// length-L circulant to the length-E one
__global__ static void k_toe_embed(float2* __restrict__ qe, const float2* __restrict__ q, GridGeom g, int E0, int E1,
		int E2, float scale)
{
	const long n = (long)E0 * E1 * E2;

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {

		int ia[3] = { (int)(i % E0), (int)((i / E0) % E1), (int)(i / ((long)E0 * E1)) };
		int E[3] = { E0, E1, E2 };
		long src = 0, stride = 1;
		bool ok = true;

		for (int a = 0; a < 3; a++) {

			int d = (ia[a] < g.N[a]) ? ia[a] : ((ia[a] > E[a] - g.N[a]) ? ia[a] - E[a] : INT_MIN);

			if (INT_MIN == d) {

				ok = false;
				break;
			}

			int j = (d < 0) ? d + g.G[a] : d;
			src += j * stride;
			stride *= g.G[a];
		}

		qe[i] = ok ? cscale(q[src], scale) : make_float2(0.f, 0.f);
	}
}

// Build p->toe / p->psf_t from p->psf (see the struct). With P the PSF on
// the L = 2N grid, the normal operator is y = sum_m x_m L q[(n - m) mod L],
// q = IDFT(P) / L per axis, and only |n - m| < N enters: on a length-E grid
// the same operator has q' = (L / E) q on |d| < N, zero elsewhere, and
// P' = DFT_E(q').
static int build_toeplitz_embedding(bnufft_plan_s* p, cudaStream_t st)
{
	const Geom& g = p->op.g;
	int E[3];
	bool embed = false;

	for (int a = 0; a < 3; a++) {

		E[a] = 1;

		if (g.G[a] > 1) {

			int e = 16;

			while (e < g.G[a])
				e *= 2;

			E[a] = e;
			embed |= (e != g.G[a]);
		}
	}

	if (p->psf_t)
		cudaFreeAsync(p->psf_t, st);

	p->psf_t = nullptr;
	p->embed = false;

	if (!embed || (E[0] > 4096) || (E[1] > 4096) || (E[2] > 4096))
		return BNUFFT_OK;

	const long L0 = g.G[0], L1 = g.G[1], L2 = g.G[2];
	const long ne = (long)E[0] * E[1] * E[2];
	float2* q = nullptr;
	float2* qe = nullptr;
	CUDA_TRY(cudaMallocAsync(&q, sizeof(float2) * g.gsz, st));
	CUDA_TRY(cudaMallocAsync(&qe, sizeof(float2) * ne, st));

	// rows of a [L0, rows] array as column-pass sequences (element stride 1),
	// at most 65535 per launch
	auto along_x = [&](int L, int mode, const float2* in, float2* out, long rows) -> int {

		for (long r0 = 0; r0 < rows; r0 += 65535) {

			long nr = std::min(65535L, rows - r0);
			TRY(cols(L, mode, in + r0 * L, 1, L, L, 0, out + r0 * L, 1, L, L, 0, 1, nr, nullptr, 0, 1, 0, st));
		}

		return BNUFFT_OK;
	};

	// unnormalised inverse DFT of the PSF along every axis (in place after the first)
	TRY(along_x((int)L0, 1, p->psf, q, L1 * L2));

	if (L1 > 1)
		TRY(cols((int)L1, 1, q, L0, L0 * L1, (int)L1, 0, q, L0, L0 * L1, (int)L1, 0, (int)L0, L2, nullptr, 0, 1, 0, st));

	if (L2 > 1)
		TRY(cols((int)L2, 1, q, L0 * L1, 0, (int)L2, 0, q, L0 * L1, 0, (int)L2, 0, (int)(L0 * L1), 1, nullptr, 0, 1, 0, st));

	k_toe_embed<<<vec_blocks(ne), RED_THREADS, 0, st>>>(qe, q, grid_geom(g), E[0], E[1], E[2], (float)(1. / (double)ne));
	LAUNCHED();

	// forward DFT on the embedding grid (powers of two)
	const long E0 = E[0], E1 = E[1], E2 = E[2];
	TRY(along_x((int)E0, 0, qe, qe, E1 * E2));

	if (E1 > 1)
		TRY(cols((int)E1, 0, qe, E0, E0 * E1, (int)E1, 0, qe, E0, E0 * E1, (int)E1, 0, (int)E0, E2, nullptr, 0, 1, 0, st));

	if (E2 > 1)
		TRY(cols((int)E2, 0, qe, E0 * E1, 0, (int)E2, 0, qe, E0 * E1, 0, (int)E2, 0, (int)(E0 * E1), 1, nullptr, 0, 1, 0, st));

	cudaFreeAsync(q, st);
	p->psf_t = qe;

	free_work(p->toe.w, st);
	p->toe = OpCtx();
	p->toe.g = g;
	p->toe.g.gsz = ne;

	for (int a = 0; a < 3; a++)
		p->toe.g.G[a] = E[a];

	p->toe.kb = p->op.kb;
	p->toe.traj = nullptr;
	p->embed = true;
	return BNUFFT_OK;
}


extern "C" void bnufft_conf_defaults(struct bnufft_conf* conf)
{
	conf->toeplitz = 1;
	conf->periodic = 0;
	conf->deterministic = 0;
	conf->os = 2.f;
	conf->width = 6.f;
	conf->bin = 0;
	conf->lowmem = 0;
}

static int check_conf(const bnufft_conf* conf)
{
	if ((0 != conf->bin) && ((conf->bin < 8) || (conf->bin > 128) || (0 != (conf->bin & (conf->bin - 1)))))
		return fail(BNUFFT_ERR_ARG, "bin edge %d (0 or a power of two 8..128)", conf->bin);

	if (!(conf->os > 1.f) || (conf->os > 4.f))
		return fail(BNUFFT_ERR_UNSUPPORTED, "oversampling %g (1 < os <= 4 is built)", conf->os);

	if ((conf->width <= 0.f) || (conf->width > 8.f))
		return fail(BNUFFT_ERR_UNSUPPORTED, "kernel width %g", conf->width);

	return BNUFFT_OK;
}

// Trajectory upload: converted trajectory and sample bins on st; with the
// Toeplitz normal the PSF chain (its own binning on the 4N grid, gridding,
// transforms, embedding) runs meanwhile on an auxiliary stream (the two are
// independent chains of small kernels). It is not joined here: p->psf_ev is
// recorded after it, and every later use of the PSF waits for that event
// (psf_wait), so work that does not need the PSF proceeds.
static int upload_traj(bnufft_plan_s* p, const void* traj, cudaStream_t st, bool own = false)
{
	Staged t;
	TRY(stage_in(t, traj, sizeof(float2) * 3 * p->op.g.M, st));

	if (own) {	// a device buffer of the caller's, freed here like a staged copy

		t.owned = true;
		t.st = st;
	}
	int dev = 0;
	CUDA_TRY(cudaGetDevice(&dev));
	const AuxStream* aux = (p->conf.toeplitz && p->psf_ev) ? aux_stream(dev) : nullptr;
	cudaStream_t pst = aux ? aux->st : st;
	int s_psf = BNUFFT_OK;
	psf_wait(p, st);	// an earlier PSF chain of this plan is done before its buffers go

	if (p->conf.toeplitz) {

		if (p->psf)
			cudaFreeAsync(p->psf, st);

		if (p->pinv)	// the preconditioner follows the PSF
			cudaFreeAsync(p->pinv, st);

		p->psf = nullptr;
		p->pinv = nullptr;

		if (aux) {

			CUDA_TRY(cudaEventRecord(aux->fork, st));
			CUDA_TRY(cudaStreamWaitEvent(pst, aux->fork, 0));
		}

		s_psf = compute_psf(p->op.g, (const float2*)t.dev, p->op.kb, &p->psf, pst, 0 != p->conf.deterministic,
				p->op.wgt, p->op.bin_edge, p->basis, p->nb, p->T, p->MrMs);

		// the block PSF of a basis stays on the 2N grid (Bluestein transforms
		// where 2N is not a power of two)
		if ((BNUFFT_OK == s_psf) && !p->nb)
			s_psf = build_toeplitz_embedding(p, pst);
	}

	k_traj_convert<<<vec_blocks(p->op.g.M), RED_THREADS, 0, st>>>(p->traj, (const float2*)t.dev, p->op.g.M, 1.f);
	cudaError_t e = cudaGetLastError();
	g_launches.fetch_add(1, std::memory_order_relaxed);
	int s = (cudaSuccess == e) ? BNUFFT_OK : fail(BNUFFT_ERR_CUDA, "trajectory: %s", cudaGetErrorString(e));
	free_bins(p->op.bins, st);

	// the chained NUFFT (os != 2) grids with the generic per-sample kernels
	if ((BNUFFT_OK == s) && !p->op.g.chain)
		s = build_bins(p->op, st);

	if ((BNUFFT_OK == s) && p->conf.deterministic) {

		free_csr(p->op.csr, st);
		s = build_csr(p->op, st);
	}

	if (p->conf.toeplitz) {	// whatever happened, so that nothing outlives its inputs

		if (p->psf_ev)
			cudaEventRecord(p->psf_ev, pst);

		if (aux) {	// the staged trajectory is freed after both streams' uses

			cudaEventRecord(aux->join, st);
			cudaStreamWaitEvent(pst, aux->join, 0);

			if (t.owned) {

				cudaFreeAsync(t.dev, pst);
				t.owned = false;
			}
		}
	}

	TRY(s_psf);
	TRY(s);

	return BNUFFT_OK;
}

extern "C" int bnufft_create2(bnufft_plan_t* plan, int N, const long ksp_dims[], const long cim_dims[],
		const long traj_dims[], const void* traj,
		const long wgh_dims[], const void* weights,
		const long bas_dims[], const void* basis,
		const struct bnufft_conf* conf_in, void* stream)
{
	*plan = nullptr;
	cudaStream_t st = S(stream);

	if ((N < 4) || (nullptr == traj))
		return fail(BNUFFT_ERR_ARG, "need N >= 4 dims and a trajectory");

	// subspace basis [1, 1, 1, 1, 1, T, K] (nufft_set_traj,
	// src/noncart/nufft.c:1018-1042): cim [X, Y, Z, ..., 1 (TE), K (COEFF)],
	// ksp [1, Mr, Ms, ..., T, 1], trajectory per frame or shared
	int nb = 0, T = 1;

	if (basis) {

		if (!bas_dims || (N < 7))
			return fail(BNUFFT_ERR_ARG, "a basis needs its dims and N >= 7");

		for (int i = 0; i < N; i++)
			if ((5 != i) && (6 != i) && (1 != bas_dims[i]))
				return fail(BNUFFT_ERR_ARG, "basis dims must be [1, 1, 1, 1, 1, T, K]");

		T = (int)bas_dims[5];
		nb = (int)bas_dims[6];

		if ((T < 1) || (nb < 1) || (nb > BASIS_MAX_K))
			return fail(BNUFFT_ERR_UNSUPPORTED, "basis with %d coefficients (at most %d)", nb, (int)BASIS_MAX_K);

		// ksp dim 6 may name the coefficients (the SENSE model passes them,
		// src/sense/modelnc.c:41-43); the k-space itself has none (out_dims,
		// src/noncart/nufft.c:1018-1022)
		if ((ksp_dims[5] != T) || ((1 != ksp_dims[6]) && (nb != ksp_dims[6])) || (1 != cim_dims[5])
				|| (cim_dims[6] != nb))
			return fail(BNUFFT_ERR_ARG, "with a basis: ksp dims 5/6 must be T/(1 or K) and image dims 5/6 1/K");

		if ((1 != traj_dims[5]) && (T != traj_dims[5]))
			return fail(BNUFFT_ERR_ARG, "trajectory frames (dim 5) must be 1 or the basis' T");
	}

	bnufft_conf conf;

	if (conf_in)
		conf = *conf_in;
	else
		bnufft_conf_defaults(&conf);

	TRY(check_conf(&conf));

	if (2.f != conf.os) {	// the chained NUFFT (src/noncart/nufft.c:1185-1198, nufft_chain.c)

		if (basis)
			return fail(BNUFFT_ERR_UNSUPPORTED, "a basis with os != 2");

		if (conf.deterministic)
			return fail(BNUFFT_ERR_UNSUPPORTED, "deterministic gridding with os != 2");

		conf.toeplitz = 0;	// the chain has no Toeplitz normal: adjoint(forward)
	}

	if (3 != traj_dims[0] || 1 != ksp_dims[0])
		return fail(BNUFFT_ERR_ARG, "traj dims[0] must be 3 and ksp dims[0] 1");

	if (ksp_dims[1] != traj_dims[1] || ksp_dims[2] != traj_dims[2])
		return fail(BNUFFT_ERR_ARG, "k-space and trajectory sample dims differ");

	for (int i = 3; i < N; i++) {

		if (nb && ((5 == i) || (6 == i)))
			continue;

		if (ksp_dims[i] != cim_dims[i])
			return fail(BNUFFT_ERR_UNSUPPORTED, "ksp/cim dim %d differ (%ld, %ld)", i, ksp_dims[i], cim_dims[i]);

		if (1 != traj_dims[i])
			return fail(BNUFFT_ERR_UNSUPPORTED, "trajectory varying along dim %d", i);
	}

	if (nb && conf.lowmem)
		return fail(BNUFFT_ERR_UNSUPPORTED, "--lowmem with a basis");

	auto p = new bnufft_plan_s();

	if (cudaSuccess != cudaEventCreateWithFlags(&p->psf_ev, cudaEventDisableTiming)) {

		cudaGetLastError();
		p->psf_ev = nullptr;	// no event: the PSF is then built on the caller's stream
	}

	p->N = N;
	p->ksp_dims.assign(ksp_dims, ksp_dims + N);
	p->cim_dims.assign(cim_dims, cim_dims + N);
	p->trj_dims.assign(traj_dims, traj_dims + N);
	p->conf = conf;
	p->C = prod(N - 3, cim_dims + 3);
	p->st0 = st;
	p->nb = nb;
	p->T = T;
	p->Cc = p->C / std::max(1, nb);
	p->MrMs = traj_dims[1] * traj_dims[2];

	long M = p->MrMs * T;	// all frames' samples
	int s = init_geom(p->op.g, cim_dims, M, conf.os, conf.width, conf.periodic);
	p->op.bin_edge = conf.bin;
	p->op.coils = conf.lowmem ? 1 : (int)std::min<long>(p->C, 1 << 20);

	if (BNUFFT_OK == s)
		s = get_kb_table(conf.os, conf.width, &p->op.kb);

	if (BNUFFT_OK == s)
		s = init_rolloff(p->op, st);

	if ((BNUFFT_OK == s) && (cudaSuccess != cudaMallocAsync(&p->traj, sizeof(float4) * M, st)))
		s = fail(BNUFFT_ERR_NOMEM, "trajectory buffer");

	p->op.traj = p->traj;

	if ((BNUFFT_OK == s) && nb) {	// the basis; weights [1, Mr, Ms, 1, 1, T or 1] over all frames' samples

		Staged bs;
		s = stage_in(bs, basis, sizeof(float2) * T * nb, st);

		if ((BNUFFT_OK == s) && (cudaSuccess != cudaMallocAsync(&p->basis, sizeof(float2) * T * nb, st)))
			s = fail(BNUFFT_ERR_NOMEM, "basis buffer");

		if ((BNUFFT_OK == s) && (cudaSuccess != cudaMemcpyAsync(p->basis, bs.dev, sizeof(float2) * T * nb, cudaMemcpyDeviceToDevice, st)))
			s = fail(BNUFFT_ERR_CUDA, "basis copy");

		if (weights && (BNUFFT_OK == s)) {

			bool ok = wgh_dims && (1 == wgh_dims[0]) && (wgh_dims[1] == ksp_dims[1]) && (wgh_dims[2] == ksp_dims[2])
				&& ((1 == wgh_dims[5]) || (T == wgh_dims[5]));

			for (int i = 3; ok && (i < N); i++)
				ok = (5 == i) || (1 == wgh_dims[i]);

			if (!ok)
				s = fail(BNUFFT_ERR_UNSUPPORTED, "with a basis, weights must be [1, Mr, Ms, 1, 1, T or 1]");

			const long wf = ok ? wgh_dims[5] : 1;	// frames the weights hold
			Staged ws;

			if (BNUFFT_OK == s)
				s = stage_in(ws, weights, sizeof(float2) * p->MrMs * wf, st);

			if ((BNUFFT_OK == s) && (cudaSuccess != cudaMallocAsync(&p->wgt, sizeof(float2) * M, st)))
				s = fail(BNUFFT_ERR_NOMEM, "weights buffer");

			for (long t = 0; (BNUFFT_OK == s) && (t < T); t++)
				if (cudaSuccess != cudaMemcpyAsync(p->wgt + p->MrMs * t, (const float2*)ws.dev + p->MrMs * (t % wf),
						sizeof(float2) * p->MrMs, cudaMemcpyDeviceToDevice, st))
					s = fail(BNUFFT_ERR_CUDA, "weights copy");

			p->op.wgt = p->wgt;
			p->op.wgt_c = 1;
		}

		if (BNUFFT_OK == s)
			cudaStreamSynchronize(st);	// the staged inputs are read before they go

		weights = nullptr;	// handled
	}

	// weights [1, Mr, Ms, 1 or C, 1...] (nufft_set_traj, src/noncart/nufft.c:1041-1049)
	if ((BNUFFT_OK == s) && weights) {

		long wc = prod(N - 3, wgh_dims + 3);

		if ((1 != wgh_dims[0]) || (wgh_dims[1] != ksp_dims[1]) || (wgh_dims[2] != ksp_dims[2]) || ((1 != wc) && (p->C != wc)))
			s = fail(BNUFFT_ERR_UNSUPPORTED, "weights must be [1, Mr, Ms] or match the k-space dims");
		else if (conf.toeplitz && (1 != wc))
			s = fail(BNUFFT_ERR_UNSUPPORTED, "per-channel weights with the Toeplitz PSF");

		if (BNUFFT_OK == s) {

			Staged ws;
			s = stage_in(ws, weights, sizeof(float2) * M * wc, st);

			if ((BNUFFT_OK == s) && (cudaSuccess != cudaMallocAsync(&p->wgt, sizeof(float2) * M * wc, st)))
				s = fail(BNUFFT_ERR_NOMEM, "weights buffer");

			if ((BNUFFT_OK == s) && (cudaSuccess != cudaMemcpyAsync(p->wgt, ws.dev, sizeof(float2) * M * wc, cudaMemcpyDeviceToDevice, st)))
				s = fail(BNUFFT_ERR_CUDA, "weights copy");

			if ((BNUFFT_OK == s) && ws.owned)
				cudaStreamSynchronize(st);

			p->op.wgt = p->wgt;
			p->op.wgt_c = wc;

			if ((BNUFFT_OK == s) && conf.lowmem && (wc > 1))
				s = fail(BNUFFT_ERR_UNSUPPORTED, "--lowmem with per-coil weights");
		}
	}

	if ((BNUFFT_OK == s) && nb && (1 == traj_dims[5]) && (T > 1)) {	// one trajectory for all frames

		float2* rep = nullptr;
		Staged ts;
		s = stage_in(ts, traj, sizeof(float2) * 3 * p->MrMs, st);

		if ((BNUFFT_OK == s) && (cudaSuccess != cudaMallocAsync(&rep, sizeof(float2) * 3 * M, st)))
			s = fail(BNUFFT_ERR_NOMEM, "trajectory frames");

		for (long t = 0; (BNUFFT_OK == s) && (t < T); t++)
			if (cudaSuccess != cudaMemcpyAsync(rep + 3 * p->MrMs * t, ts.dev, sizeof(float2) * 3 * p->MrMs,
					cudaMemcpyDeviceToDevice, st))
				s = fail(BNUFFT_ERR_CUDA, "trajectory frames");

		if (BNUFFT_OK == s)
			s = upload_traj(p, rep, st, true);
		else if (rep)
			cudaFreeAsync(rep, st);

	} else if (BNUFFT_OK == s) {

		s = upload_traj(p, traj, st);
	}

	if (BNUFFT_OK != s) {

		std::string msg = g_err;
		bnufft_free(p);
		g_err = msg;
		return s;
	}

	*plan = p;
	return BNUFFT_OK;
}

extern "C" int bnufft_update_traj(bnufft_plan_t p, int N, const long traj_dims[], const void* traj, void* stream)
{
	if (!p || (N != p->N))
		return fail(BNUFFT_ERR_ARG, "bad plan or dims");

	if (p->nb)
		return fail(BNUFFT_ERR_UNSUPPORTED, "trajectory update of a plan with a basis");

	for (int i = 0; i < N; i++)
		if (traj_dims[i] != p->trj_dims[i])
			return fail(BNUFFT_ERR_ARG, "trajectory dims changed (dim %d)", i);

	return upload_traj(p, traj, S(stream));
}

// coils per apply pass: all, or one with --lowmem (the work grids then hold
// one coil; results are the same)
static long coil_chunk(const bnufft_plan_s* p) { return p->conf.lowmem ? 1 : p->C; }

// forward / adjoint with a subspace basis: the NUFFT of every (coil,
// coefficient) channel at all frames' samples, then the basis contraction
// over the coefficients (nufft_apply_forward, src/noncart/nufft.c:1443-1453;
// the adjoint expands with conj(B) first, :1483-1487)
static int basis_forward(bnufft_plan_s* p, const float2* x, float2* y, cudaStream_t st)
{
	const long M = p->op.g.M;
	float2* tmp = nullptr;
	CUDA_TRY(cudaMallocAsync(&tmp, sizeof(float2) * M * p->C, st));
	int s = op_forward(p->op, x, nullptr, p->C, tmp, st);

	if (BNUFFT_OK == s) {

		k_basis_contract<<<vec_blocks(M * p->Cc), RED_THREADS, 0, st>>>(y, tmp, p->basis, p->MrMs, p->T, p->Cc, p->nb);
		cudaError_t e = cudaGetLastError();
		g_launches.fetch_add(1, std::memory_order_relaxed);
		s = (cudaSuccess == e) ? BNUFFT_OK : fail(BNUFFT_ERR_CUDA, "basis contraction: %s", cudaGetErrorString(e));
	}

	cudaFreeAsync(tmp, st);
	return s;
}

static int basis_adjoint(bnufft_plan_s* p, const float2* y, float2* x, cudaStream_t st)
{
	const long M = p->op.g.M;
	float2* tmp = nullptr;
	CUDA_TRY(cudaMallocAsync(&tmp, sizeof(float2) * M * p->C, st));
	k_basis_expand<<<vec_blocks(M * p->C), RED_THREADS, 0, st>>>(tmp, y, p->basis, p->MrMs, p->T, p->Cc, p->nb);
	cudaError_t e = cudaGetLastError();
	g_launches.fetch_add(1, std::memory_order_relaxed);
	int s = (cudaSuccess == e) ? op_adjoint(p->op, tmp, nullptr, p->C, 1, x, st)
				: fail(BNUFFT_ERR_CUDA, "basis expansion: %s", cudaGetErrorString(e));
	cudaFreeAsync(tmp, st);
	return s;
}

extern "C" int bnufft_apply_forward(bnufft_plan_t p, void* dst, const void* src, void* stream)
{
	cudaStream_t st = S(stream);
	const long npix = p->op.g.npix, M = p->op.g.M, cc = coil_chunk(p);
	size_t in_b = sizeof(float2) * npix * p->C;
	size_t out_b = sizeof(float2) * M * (p->nb ? p->Cc : p->C);
	Staged i, o;
	TRY(stage_in(i, src, in_b, st));
	TRY(stage_out_alloc(o, dst, out_b, st));

	if (p->nb) {

		TRY(basis_forward(p, (const float2*)i.dev, (float2*)o.dev, st));
		return stage_out_copy(o, dst, out_b, st);
	}

	for (long c0 = 0; c0 < p->C; c0 += cc)
		TRY(op_forward(p->op, (const float2*)i.dev + npix * c0, nullptr, std::min(cc, p->C - c0),
				(float2*)o.dev + M * c0, st));

	return stage_out_copy(o, dst, out_b, st);
}

extern "C" int bnufft_apply_adjoint(bnufft_plan_t p, void* dst, const void* src, void* stream)
{
	cudaStream_t st = S(stream);
	const long npix = p->op.g.npix, M = p->op.g.M, cc = coil_chunk(p);
	size_t in_b = sizeof(float2) * M * (p->nb ? p->Cc : p->C);
	size_t out_b = sizeof(float2) * npix * p->C;
	Staged i, o;
	TRY(stage_in(i, src, in_b, st));
	TRY(stage_out_alloc(o, dst, out_b, st));

	if (p->nb) {

		TRY(basis_adjoint(p, (const float2*)i.dev, (float2*)o.dev, st));
		return stage_out_copy(o, dst, out_b, st);
	}

	for (long c0 = 0; c0 < p->C; c0 += cc)
		TRY(op_adjoint(p->op, (const float2*)i.dev + M * c0, nullptr, std::min(cc, p->C - c0), 1,
				(float2*)o.dev + npix * c0, st));

	return stage_out_copy(o, dst, out_b, st);
}

extern "C" int bnufft_apply_normal(bnufft_plan_t p, void* dst, const void* src, void* stream)
{
	cudaStream_t st = S(stream);
	size_t b = sizeof(float2) * p->op.g.npix * p->C;
	Staged i, o;
	TRY(stage_in(i, src, b, st));
	TRY(stage_out_alloc(o, dst, b, st));

	if (p->nb) {	// block-Toeplitz, or the adjoint of the forward

		if (p->psf) {

			psf_wait(p, st);
			TRY(op_toeplitz_basis(p->op, p->psf, (const float2*)i.dev, p->Cc, p->nb, (float2*)o.dev, st));

		} else {

			float2* k = nullptr;
			CUDA_TRY(cudaMallocAsync(&k, sizeof(float2) * p->op.g.M * p->Cc, st));
			int s = basis_forward(p, (const float2*)i.dev, k, st);

			if (BNUFFT_OK == s)
				s = basis_adjoint(p, k, (float2*)o.dev, st);

			cudaFreeAsync(k, st);
			TRY(s);
		}

		return stage_out_copy(o, dst, b, st);
	}

	if (p->psf) {

		const long npix = p->op.g.npix, cc = coil_chunk(p);

		for (long c0 = 0; c0 < p->C; c0 += cc)
			TRY(op_toeplitz(toe_ctx(p), toe_psf(p, st), (const float2*)i.dev + npix * c0, nullptr, std::min(cc, p->C - c0),
					1, (float2*)o.dev + npix * c0, st));

	} else {

		float2* k = nullptr;
		CUDA_TRY(cudaMallocAsync(&k, sizeof(float2) * p->op.g.M * p->C, st));
		TRY(op_forward(p->op, (const float2*)i.dev, nullptr, p->C, k, st));
		TRY(op_adjoint(p->op, k, nullptr, p->C, 1, (float2*)o.dev, st));
		cudaFreeAsync(k, st);
	}

	return stage_out_copy(o, dst, b, st);
}

extern "C" int bnufft_get_psf_dims(bnufft_plan_t p, int ND, long psf_dims[])
{
	if (!p || !p->psf)
		return fail(BNUFFT_ERR_ARG, "plan has no PSF");

	if (p->nb)
		return fail(BNUFFT_ERR_UNSUPPORTED, "the block PSF of a basis in the decomposed layout");

	if (ND != p->N + 1)
		return fail(BNUFFT_ERR_ARG, "PSF has N+1 = %d dims", p->N + 1);

	for (int i = 0; i < ND; i++)
		psf_dims[i] = 1;

	long sub = 1;

	for (int i = 0; i < 3; i++) {

		psf_dims[i] = p->op.g.N[i];
		sub *= (p->op.g.G[i] > 1) ? 2 : 1;
	}

	psf_dims[p->N] = sub;
	return BNUFFT_OK;
}

// decomposed layout of the reference: psf[w + N*..., s] = P_centred[2w + s] * npix
__global__ static void k_psf_decompose(float2* dst, const float2* psf, GridGeom g, float npix)
{
	long n = (long)g.N[0] * g.N[1] * g.N[2];
	long tot = n * ((g.G[0] > 1 ? 2 : 1) * (g.G[1] > 1 ? 2 : 1) * (g.G[2] > 1 ? 2 : 1));

	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += (long)gridDim.x * blockDim.x) {

		long pix = i % n;
		long sidx = i / n;
		int w[3] = { (int)(pix % g.N[0]), (int)((pix / g.N[0]) % g.N[1]), (int)(pix / ((long)g.N[0] * g.N[1])) };
		long cell = 0;
		long stride = 1;

		for (int a = 0; a < 3; a++) {

			int s = 0;

			if (g.G[a] > 1) {

				s = (int)(sidx & 1);
				sidx >>= 1;
			}

			int j = (g.G[a] > 1) ? (2 * w[a] + s + g.N[a]) % g.G[a] : 0;
			cell += j * stride;
			stride *= g.G[a];
		}

		dst[i] = cscale(psf[cell], npix);
	}
}

extern "C" int bnufft_get_psf(bnufft_plan_t p, int ND, const long psf_dims[], void* psf, void* stream)
{
	long d[32];

	if (ND > 32)
		return fail(BNUFFT_ERR_ARG, "too many dims");

	TRY(bnufft_get_psf_dims(p, ND, d));

	for (int i = 0; i < ND; i++)
		if (d[i] != psf_dims[i])
			return fail(BNUFFT_ERR_ARG, "PSF dim %d is %ld, not %ld", i, d[i], psf_dims[i]);

	cudaStream_t st = S(stream);
	size_t b = sizeof(float2) * p->op.g.gsz;
	Staged o;
	TRY(stage_out_alloc(o, psf, b, st));
	psf_wait(p, st);
	k_psf_decompose<<<vec_blocks(p->op.g.gsz), RED_THREADS, 0, st>>>((float2*)o.dev, p->psf, grid_geom(p->op.g), (float)p->op.g.npix);
	LAUNCHED();
	return stage_out_copy(o, psf, b, st);
}

extern "C" void bnufft_free(bnufft_plan_t p)
{
	if (!p)
		return;

	cudaStream_t st = p->st0;
	psf_wait(p, st);	// the frees follow the auxiliary stream's work on the PSF
	free_work(p->op.w, st);
	free_work(p->toe.w, st);
	free_csr(p->op.csr, st);
	free_bins(p->op.bins, st);

	if (p->traj) cudaFreeAsync(p->traj, st);
	if (p->psf) cudaFreeAsync(p->psf, st);
	if (p->psf_t) cudaFreeAsync(p->psf_t, st);
	if (p->wgt) cudaFreeAsync(p->wgt, st);
	if (p->pinv) cudaFreeAsync(p->pinv, st);
	if (p->op.wbuf) cudaFreeAsync(p->op.wbuf, st);
	if (p->basis) cudaFreeAsync(p->basis, st);

	if (p->psf_ev)
		cudaEventDestroy(p->psf_ev);

	delete p;	// device frees are stream-ordered; host state can go now
}

// ----------------------------------------------------------------------------
// nufft -i: CG over coil images, optional circulant preconditioner
// ----------------------------------------------------------------------------

// Circulant preconditioner of the Toeplitz normal (nufft_precond_create,
// src/noncart/precond.c:36-64, 95-130). Its kernel is the central N-cell part
// of the PSF's image-domain kernel h; the reference assembles it from the 2^d
// decomposed sub-grids with their linear phases, which equals 2^d h(x - N/2)
// and, through the fftmod factor in those phases, leaves the spectrum in
// uncentred order. Here: crop = unnormalised inverse 2N transform of the PSF
// (DFT order, already 1/npix) with the central crop (= 2^d h), forward
// N-point transform with the centred placement, pre = |.|/sqrt(npix) + 1e-3.
static int build_precond(bnufft_plan_s* p, cudaStream_t st)
{
	if (p->pinv)
		return BNUFFT_OK;

	if (!p->psf)
		return fail(BNUFFT_ERR_ARG, "the circulant preconditioner needs the Toeplitz PSF");

	psf_wait(p, st);
	// work buffers of its own: it may run on the auxiliary stream while the
	// plan's buffers serve the solve on another stream
	OpCtx op = p->op;
	op.w = Work{};
	const Geom& g = op.g;
	TRY(alloc_work(op.w, g, 1, st));
	float2* crop = nullptr;
	float2* F = nullptr;
	CUDA_TRY(cudaMallocAsync(&crop, sizeof(float2) * g.npix, st));
	CUDA_TRY(cudaMallocAsync(&F, sizeof(float2) * g.npix, st));
	TRY(op_spectrum_adjoint(op, p->psf, nullptr, false, 1, 1, crop, st));

	// forward N-point transform (no zero padding): a geometry with L = N
	OpCtx full;
	full.g = g;

	for (int a = 0; a < 3; a++)
		full.g.G[a] = g.N[a];

	full.g.gsz = g.npix;
	full.kb = op.kb;
	full.traj = nullptr;
	TRY(alloc_work(full.w, full.g, 1, st));
	TRY(op_spectrum(full, crop, nullptr, false, 1, F, st));
	CUDA_TRY(cudaMallocAsync(&p->pinv, sizeof(float2) * g.npix, st));
	k_precond_from_spectrum<<<vec_blocks(g.npix), RED_THREADS, 0, st>>>(p->pinv, F, g.npix, (float)(1. / sqrt((double)g.npix)));
	LAUNCHED();
	free_work(full.w, st);
	free_work(op.w, st);
	cudaFreeAsync(crop, st);
	cudaFreeAsync(F, st);
	return BNUFFT_OK;
}

// v <- P^-1 v = ifft(fft(v) / pre) per coil (uncentred, unnormalised)
static int apply_precond(bnufft_plan_s* p, float2* v, long C, cudaStream_t st)
{
	OpCtx full;
	full.g = p->op.g;

	for (int a = 0; a < 3; a++)
		full.g.G[a] = full.g.N[a];

	full.g.gsz = full.g.npix;
	full.kb = p->op.kb;
	full.traj = nullptr;
	full.w = p->op.w;	// borrow the plan's buffers (large enough: N <= 2N)
	const Geom& g = full.g;
	long YZ = (long)g.N[1] * g.N[2];
	TRY(rows_fwd(g.G[0], v, nullptr, nullptr, nullptr, g.N[0], YZ, YZ * C, full.w.t1, st));
	TRY(op_toeplitz_cols(full, precond_spec(p, st), C, st));
	return rows_inv(g.G[0], full.w.t1, nullptr, nullptr, nullptr, g.N[0], YZ, (int)C, 1, v, st);
}

extern "C" int bnufft_nufft_inverse(bnufft_plan_t p, void* img, const void* ksp, float lambda, int maxiter,
		int precond, void* stream)
{
	cudaStream_t st = S(stream);

	if (!p || (maxiter < 0))
		return fail(BNUFFT_ERR_ARG, "bad plan or iteration count");

	if (p->nb)
		return fail(BNUFFT_ERR_UNSUPPORTED, "nufft -i with a basis");

	OpCtx& op = p->op;
	const long C = p->C;
	const long n = op.g.npix * C;
	size_t kb = sizeof(float2) * op.g.M * C;
	size_t ib = sizeof(float2) * n;
	Staged ki, io;
	TRY(stage_in(ki, ksp, kb, st));
	TRY(stage_out_alloc(io, img, ib, st));
	float2* x = (float2*)io.dev;

	if (precond)
		TRY(build_precond(p, st));

	float2 *r = nullptr, *pv = nullptr, *Ap = nullptr;
	double *pap = nullptr, *rsp = nullptr;
	CgScalars* sc = nullptr;
	unsigned nb = vec_blocks(n);
	CUDA_TRY(cudaMallocAsync(&r, ib, st));
	CUDA_TRY(cudaMallocAsync(&pv, ib, st));
	CUDA_TRY(cudaMallocAsync(&Ap, ib, st));
	CUDA_TRY(cudaMallocAsync(&pap, sizeof(double) * nb, st));
	CUDA_TRY(cudaMallocAsync(&rsp, sizeof(double) * nb, st));
	CUDA_TRY(cudaMallocAsync(&sc, sizeof(CgScalars), st));

	// b = P^-1 N^H y  (into r, then CG start from x = 0)
	TRY(op_adjoint(op, (const float2*)ki.dev, nullptr, C, 1, Ap, st));

	if (precond)
		TRY(apply_precond(p, Ap, C, st));

	k_cg_init<<<nb, RED_THREADS, 0, st>>>(x, r, pv, Ap, n, rsp);
	LAUNCHED();
	k_cg_start<<<1, RED_THREADS, 0, st>>>(sc, rsp, (int)nb, 0.f, maxiter, 1);
	LAUNCHED();

	for (int it = 0; it < maxiter; it++) {

		// Ap = P^-1 (N^H N p + lambda p); partial p^H Ap
		if (p->psf) {

			TRY(op_toeplitz(toe_ctx(p), toe_psf(p, st), pv, nullptr, C, 1, Ap, st));

		} else {

			float2* k = nullptr;
			CUDA_TRY(cudaMallocAsync(&k, kb, st));
			TRY(op_forward(op, pv, nullptr, C, k, st));
			TRY(op_adjoint(op, k, nullptr, C, 1, Ap, st));
			cudaFreeAsync(k, st);
		}

		k_combine<<<nb, RED_THREADS, 0, st>>>(Ap, Ap, 1, n, pv, lambda, nullptr, &sc->done);
		LAUNCHED();

		if (precond)
			TRY(apply_precond(p, Ap, C, st));

		k_combine<<<nb, RED_THREADS, 0, st>>>(Ap, Ap, 1, n, pv, 0.f, pap, &sc->done);
		LAUNCHED();
		k_cg_step<<<nb, RED_THREADS, 0, st>>>(x, r, pv, Ap, 1, n, 0.f, sc, it, pap, (int)nb, nullptr, 0, rsp, nullptr);
		LAUNCHED();
		k_cg_dir<<<nb, RED_THREADS, 0, st>>>(pv, r, n, sc, it, rsp, (int)nb);
		LAUNCHED();
	}

	void* frees[] = { r, pv, Ap, pap, rsp, sc };

	for (void* q : frees)
		cudaFreeAsync(q, st);

	return stage_out_copy(io, img, ib, st);
}

// ----------------------------------------------------------------------------
// CG-SENSE (C ABI)
// ----------------------------------------------------------------------------

// ----------------------------------------------------------------------------
// direct non-uniform DFT (C ABI: bnufft_nudft_*)
// ----------------------------------------------------------------------------

struct bnufft_nudft_s {

	NudftGeom g;
	float4* traj = nullptr;		// [M] (kx, ky, kz, 0)
	cudaStream_t st0 = nullptr;
};

extern "C" void bnufft_nudft_free(bnufft_nudft_t p)
{
	if (!p)
		return;

	if (p->traj)
		cudaFreeAsync(p->traj, p->st0);

	delete p;
}

extern "C" int bnufft_nudft_create(bnufft_nudft_t* out, int N, const long ksp_dims[], const long cim_dims[],
		const long traj_dims[], const void* traj, void* stream)
{
	cudaStream_t st = S(stream);

	if (!out || !ksp_dims || !cim_dims || !traj_dims || !traj || (N < 4))
		return fail(BNUFFT_ERR_ARG, "null argument or fewer than 4 dims");

	if ((3 != traj_dims[0]) || (1 != ksp_dims[0]) || (ksp_dims[1] != traj_dims[1]) || (ksp_dims[2] != traj_dims[2]))
		return fail(BNUFFT_ERR_ARG, "trajectory [3, Mr, Ms] and k-space [1, Mr, Ms, ...] do not match");

	for (int i = 3; i < N; i++)
		if ((i < N) && (traj_dims[i] != 1))
			return fail(BNUFFT_ERR_UNSUPPORTED, "trajectory with dims beyond 2");

	long C = prod(N - 3, cim_dims + 3);

	if (prod(N - 3, ksp_dims + 3) != C)
		return fail(BNUFFT_ERR_ARG, "k-space and image batch dims differ");

	auto p = new bnufft_nudft_s();
	p->st0 = st;

	for (int a = 0; a < 3; a++)
		p->g.N[a] = (int)cim_dims[a];

	p->g.npix = (long)cim_dims[0] * cim_dims[1] * cim_dims[2];
	p->g.M = traj_dims[1] * traj_dims[2];
	p->g.C = C;
	// the reference scales by all image dims, coils included (nudft_forward2,
	// src/noncart/nudft.c:122-124)
	p->g.scale = (float)(1. / sqrt((double)(p->g.npix * C)));

	Staged t;
	int s = stage_in(t, traj, sizeof(float2) * 3 * p->g.M, st);
	cudaError_t e = cudaSuccess;

	if (BNUFFT_OK == s)
		e = cudaMallocAsync(&p->traj, sizeof(float4) * p->g.M, st);

	if ((BNUFFT_OK == s) && (cudaSuccess != e))
		s = fail(BNUFFT_ERR_NOMEM, "nudft trajectory: %s", cudaGetErrorString(e));

	if (BNUFFT_OK == s) {

		k_traj_convert<<<vec_blocks(p->g.M), RED_THREADS, 0, st>>>(p->traj, (const float2*)t.dev, p->g.M, 1.f);
		e = cudaGetLastError();
		g_launches.fetch_add(1, std::memory_order_relaxed);

		if (cudaSuccess != e)
			s = fail(BNUFFT_ERR_CUDA, "nudft trajectory: %s", cudaGetErrorString(e));
	}

	if ((BNUFFT_OK == s) && t.owned)
		e = cudaStreamSynchronize(st);

	if (BNUFFT_OK != s) {

		std::string msg = g_err;
		bnufft_nudft_free(p);
		g_err = msg;
		return s;
	}

	*out = p;
	return BNUFFT_OK;
}

extern "C" int bnufft_nudft_apply_forward(bnufft_nudft_t p, void* ksp, const void* cim, void* stream)
{
	cudaStream_t st = S(stream);
	const NudftGeom& g = p->g;
	Staged i, o;
	TRY(stage_in(i, cim, sizeof(float2) * g.npix * g.C, st));
	TRY(stage_out_alloc(o, ksp, sizeof(float2) * g.M * g.C, st));
	dim3 grid((unsigned)((g.M + NUDFT_THREADS - 1) / NUDFT_THREADS), (unsigned)((g.C + NUDFT_CC - 1) / NUDFT_CC));
	k_nudft_fwd<<<grid, NUDFT_THREADS, 0, st>>>(p->traj, g, (const float2*)i.dev, (float2*)o.dev);
	LAUNCHED();
	return stage_out_copy(o, ksp, sizeof(float2) * g.M * g.C, st);
}

extern "C" int bnufft_nudft_apply_adjoint(bnufft_nudft_t p, void* cim, const void* ksp, void* stream)
{
	cudaStream_t st = S(stream);
	const NudftGeom& g = p->g;
	Staged i, o;
	TRY(stage_in(i, ksp, sizeof(float2) * g.M * g.C, st));
	TRY(stage_out_alloc(o, cim, sizeof(float2) * g.npix * g.C, st));
	dim3 grid((unsigned)((g.npix + NUDFT_THREADS - 1) / NUDFT_THREADS), (unsigned)((g.C + NUDFT_CC - 1) / NUDFT_CC));
	k_nudft_adj<<<grid, NUDFT_THREADS, 0, st>>>(p->traj, g, (const float2*)i.dev, (float2*)o.dev);
	LAUNCHED();
	return stage_out_copy(o, cim, sizeof(float2) * g.npix * g.C, st);
}

// ----------------------------------------------------------------------------
// learned preconditioner network (C ABI: bnufft_precnet_*)
// ----------------------------------------------------------------------------

struct bnufft_precnet_s {

	float* params = nullptr;	// float32 master parameters
	float* pr = nullptr;		// working copy: weights rounded to bf16, biases float
	bf16* wf = nullptr;		// layers 2-5 forward weights [4][32][9][32]
	bf16* wt = nullptr;		// layers 2-5 transposed, tap-flipped [4][32][9][32]
	float *m = nullptr, *v = nullptr, *grad = nullptr;	// Adam moments, gradient
	int step = 0;
	// training workspace, sized for P pixels and nblk tiles
	long ws_P = 0, ws_nblk = 0;
	bf16* act[5] = { nullptr, nullptr, nullptr, nullptr, nullptr };
	bf16 *gu0 = nullptr, *gu1 = nullptr;
	float2 *out = nullptr, *gout = nullptr;
	float* part = nullptr;
	double* loss_part = nullptr;
	double* loss_host = nullptr;	// pinned
	int* tc_status = nullptr;	// tensor-core conv error word (1: a wait ran out)
	bf16* wf_tc = nullptr;		// wf and wt in the tensor-core kernel's B-plane order
	bf16* wt_tc = nullptr;
};

static const int NET_N = NetLayout::total();
enum { NET_LOSS_BLOCKS = 256 };

static int net_pack(bnufft_precnet_s* n, cudaStream_t st)
{
	k_net_pack<<<(NET_N + 255) / 256, 256, 0, st>>>(n->params, n->pr, n->wf, n->wt);
	LAUNCHED();
	k_net_pack_tc<<<(4 * 9216 + 255) / 256, 256, 0, st>>>(n->wf, n->wf_tc);
	LAUNCHED();
	k_net_pack_tc<<<(4 * 9216 + 255) / 256, 256, 0, st>>>(n->wt, n->wt_tc);
	LAUNCHED();
	return BNUFFT_OK;
}

static dim3 net_tiles(int X, int Y, long nimg)
{
	return dim3((unsigned)((X + NET_TILE_X - 1) / NET_TILE_X), (unsigned)((Y + NET_TILE_Y - 1) / NET_TILE_Y), (unsigned)nimg);
}

// cuTensorMapEncodeTiled from the driver (no link against libcuda)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
	static std::once_flag once;
	static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
	std::call_once(once, [] {
		void* p = nullptr;
		cudaDriverEntryPointQueryResult q;

		if ((cudaSuccess == cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q))
				&& (cudaDriverEntryPointSuccess == q))
			fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
	});
	return fn;
}

static int sm_count()
{
	int dev, n = 0;
	CUDA_TRY(cudaGetDevice(&dev));
	CUDA_TRY(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
	return n;
}

// One 32 -> 32 layer: the tcgen05 kernel (default; work tiles of two rows
// of 128 pixels) or the mma.sync kernel (BNUFFT_NET_TC=0). wtc: the layer's
// weights in the tensor-core kernel's plane order; w: the same in the
// mma.sync kernel's order.
template <int MODE>
static int launch_conv32(const bnufft_precnet_s* n, const bf16* in, const bf16* w, const bf16* wtc,
		const float* bias, const bf16* mask, bf16* out, int X, int Y, long nimg, const int* done, const int* skip,
		cudaStream_t st)
{
	const char* e = getenv("BNUFFT_NET_TC");
	constexpr int R = 2;

	if (!(e && (0 == strcmp(e, "0")))) {

		auto enc = tensor_map_encoder();

		if (!enc)
			return fail(BNUFFT_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");

		// activations [nimg][Y][X][32] bf16; box {8 channels, 130 pixels, R + 2 rows, 1 image}
		CUtensorMap map;
		const cuuint64_t gdim[4] = { (cuuint64_t)NET_C, (cuuint64_t)X, (cuuint64_t)Y, (cuuint64_t)nimg };
		const cuuint64_t gstr[3] = { (cuuint64_t)NET_C * 2, (cuuint64_t)NET_C * 2 * X, (cuuint64_t)NET_C * 2 * X * Y };
		const cuuint32_t box[4] = { 8, TC_HX, R + 2, 1 };
		const cuuint32_t estr[4] = { 1, 1, 1, 1 };
		CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void*)in, gdim, gstr, box, estr,
				CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
				CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);

		if (CUDA_SUCCESS != r)
			return fail(BNUFFT_ERR_CUDA, "cuTensorMapEncodeTiled: error %d", (int)r);

		const size_t smem = conv_tc_smem(R);
		TRY(prep_kernel(k_conv32_tc<MODE, R>, smem));
		const long tiles = (long)((X + TC_M - 1) / TC_M) * ((Y + R - 1) / R) * nimg;
		const int per_sm = (int)std::max<size_t>(1, (227 * 1024) / (smem + 1024));
		const long blocks = std::min<long>(tiles, (long)sm_count() * std::min(per_sm, 4));
		k_conv32_tc<MODE, R><<<(unsigned)blocks, 128, smem, st>>>(map, wtc, bias, mask, out, X, Y, (int)nimg, done,
				skip, n->tc_status);
		LAUNCHED();
		return BNUFFT_OK;
	}

	TRY(prep_kernel(k_conv32<MODE>, NET_CONV_SMEM));
	k_conv32<MODE><<<net_tiles(X, Y, nimg), NET_THREADS, NET_CONV_SMEM, st>>>(in, w, bias, mask, out, X, Y, done,
			skip);
	LAUNCHED();
	return BNUFFT_OK;
}

// Forward through all six layers: act[0..4] (layer 1-5 outputs, bf16) and
// out = zc + scale_out * net(scale_in * in). acts may alias in pairs for
// inference (acts[i] != acts[i - 1]). scale_in null: the input's own norm
// from in_norm_part (if given); scale_out null: the norm of zc from
// norm_part. With *net_off the layers do nothing and out = zc.
static int net_forward(const bnufft_precnet_s* n, const float2* in, int X, int Y, long nimg, bf16* const acts[5],
		const float* scale_in, const float* scale_out, const double* norm_part, int nnorm, const float2* zc,
		float2* out, const float2* pdot, double* dot_part, int* nblocks, const int* done, const int* net_off,
		cudaStream_t st, const double* in_norm_part = nullptr, int in_nnorm = 0)
{
	const long P = (long)X * Y * nimg;
	const unsigned pb = (unsigned)((P + NET_THREADS - 1) / NET_THREADS);
	const float* pr = n->pr;

	k_net_in<<<pb, NET_THREADS, 0, st>>>(in, X, Y, P, pr + NetLayout::woff(0), pr + NetLayout::boff(0), scale_in,
			in_norm_part, in_nnorm, acts[0], done, net_off);
	LAUNCHED();

	for (int l = 1; l <= 4; l++) {

		TRY(launch_conv32<0>(n, acts[l - 1], n->wf + (l - 1) * 9216, n->wf_tc + (l - 1) * 9216, pr + NetLayout::boff(l),
				nullptr, acts[l], X, Y, nimg, done, net_off, st));
	}

	k_net_out<<<pb, NET_THREADS, 0, st>>>(acts[4], X, Y, P, pr + NetLayout::woff(5), pr + NetLayout::boff(5), scale_out,
			norm_part, nnorm, zc, out, pdot, dot_part, done, net_off);
	LAUNCHED();

	if (nblocks)
		*nblocks = (int)pb;

	return BNUFFT_OK;
}

static void net_free_ws(bnufft_precnet_s* n)
{
	void* bufs[] = { n->act[0], n->act[1], n->act[2], n->act[3], n->act[4], n->gu0, n->gu1, n->out, n->gout, n->part,
			 n->loss_part };

	for (void* b : bufs)
		if (b)
			cudaFree(b);

	for (auto& a : n->act)
		a = nullptr;

	n->gu0 = n->gu1 = nullptr;
	n->out = n->gout = nullptr;
	n->part = nullptr;
	n->loss_part = nullptr;
	n->ws_P = n->ws_nblk = 0;
}

static int net_ensure_ws(bnufft_precnet_s* n, long P, long nblk)
{
	if ((P <= n->ws_P) && (nblk <= n->ws_nblk))
		return BNUFFT_OK;

	CUDA_TRY(cudaDeviceSynchronize());	// buffers may be in use by earlier steps
	net_free_ws(n);
	size_t ab = sizeof(bf16) * NET_C * P;

	for (auto& a : n->act)
		CUDA_TRY(cudaMalloc(&a, ab));

	CUDA_TRY(cudaMalloc(&n->gu0, ab));
	CUDA_TRY(cudaMalloc(&n->gu1, ab));
	CUDA_TRY(cudaMalloc(&n->out, sizeof(float2) * P));
	CUDA_TRY(cudaMalloc(&n->gout, sizeof(float2) * P));
	CUDA_TRY(cudaMalloc(&n->part, sizeof(float) * nblk * NetLayout::size(1)));
	CUDA_TRY(cudaMalloc(&n->loss_part, sizeof(double) * NET_LOSS_BLOCKS));
	n->ws_P = P;
	n->ws_nblk = nblk;
	return BNUFFT_OK;
}

// weight and bias gradients of layer l into grad
template <int CIN, int COUT, typename AT, typename GT>
static int net_wgrad(bnufft_precnet_s* n, int l, const AT* a, const GT* g, int X, int Y, long nimg, cudaStream_t st)
{
	size_t smem = sizeof(float) * (NET_HALO_Y * NET_HALO_X * CIN + NET_TILE_Y * NET_TILE_X * COUT);
	dim3 grid = net_tiles(X, Y, nimg);
	long nblk = (long)grid.x * grid.y * grid.z;
	const int O = COUT * 9 * CIN + COUT;
	TRY(prep_kernel(k_wgrad<CIN, COUT, AT, GT>, smem));
	k_wgrad<CIN, COUT, AT, GT><<<grid, NET_THREADS, smem, st>>>(a, g, X, Y, n->part);
	LAUNCHED();
	k_wgrad_reduce<<<(O + 255) / 256, 256, 0, st>>>(n->part, nblk, O, n->grad + NetLayout::woff(l));
	LAUNCHED();
	return BNUFFT_OK;
}

extern "C" int bnufft_precnet_nparams(void) { return NET_N; }

extern "C" int bnufft_precnet_set_params(bnufft_precnet_t n, const float* params, void* stream)
{
	cudaStream_t st = S(stream);
	CUDA_TRY(cudaMemcpyAsync(n->params, params, sizeof(float) * NET_N, cudaMemcpyDefault, st));
	CUDA_TRY(cudaMemsetAsync(n->m, 0, sizeof(float) * NET_N, st));
	CUDA_TRY(cudaMemsetAsync(n->v, 0, sizeof(float) * NET_N, st));
	n->step = 0;
	return net_pack(n, st);
}

extern "C" int bnufft_precnet_get_params(bnufft_precnet_t n, float* params, void* stream)
{
	cudaStream_t st = S(stream);
	CUDA_TRY(cudaMemcpyAsync(params, n->params, sizeof(float) * NET_N, cudaMemcpyDefault, st));
	CUDA_TRY(cudaStreamSynchronize(st));
	return BNUFFT_OK;
}

extern "C" int bnufft_precnet_status(bnufft_precnet_t n, int* status, void* stream)
{
	if (!n || !status)
		return fail(BNUFFT_ERR_ARG, "null argument");

	cudaStream_t st = S(stream);
	CUDA_TRY(cudaMemcpyAsync(status, n->tc_status, sizeof(int), cudaMemcpyDeviceToHost, st));
	CUDA_TRY(cudaStreamSynchronize(st));
	return BNUFFT_OK;
}

extern "C" void bnufft_precnet_free(bnufft_precnet_t n)
{
	if (!n)
		return;

	cudaDeviceSynchronize();
	net_free_ws(n);
	void* bufs[] = { n->params, n->pr, n->wf, n->wt, n->m, n->v, n->grad, n->tc_status, n->wf_tc, n->wt_tc };

	for (void* b : bufs)
		if (b)
			cudaFree(b);

	if (n->loss_host)
		cudaFreeHost(n->loss_host);

	delete n;
}

extern "C" int bnufft_precnet_create(bnufft_precnet_t* out, const float* params, void* stream)
{
	if (!out || !params)
		return fail(BNUFFT_ERR_ARG, "null argument");

	auto n = new bnufft_precnet_s();
	cudaError_t e = cudaSuccess;
	auto al = [&](void** p, size_t b) { if (cudaSuccess == e) e = cudaMalloc(p, b); };
	al((void**)&n->params, sizeof(float) * NET_N);
	al((void**)&n->pr, sizeof(float) * NET_N);
	al((void**)&n->m, sizeof(float) * NET_N);
	al((void**)&n->v, sizeof(float) * NET_N);
	al((void**)&n->grad, sizeof(float) * NET_N);
	al((void**)&n->wf, sizeof(bf16) * 4 * 9216);
	al((void**)&n->wt, sizeof(bf16) * 4 * 9216);
	al((void**)&n->tc_status, sizeof(int));
	al((void**)&n->wf_tc, sizeof(bf16) * 4 * 9216);
	al((void**)&n->wt_tc, sizeof(bf16) * 4 * 9216);

	if (cudaSuccess == e)
		e = cudaMemset(n->tc_status, 0, sizeof(int));

	if (cudaSuccess == e)
		e = cudaMallocHost((void**)&n->loss_host, sizeof(double) * NET_LOSS_BLOCKS);

	if (cudaSuccess != e) {

		bnufft_precnet_free(n);
		return fail(BNUFFT_ERR_NOMEM, "precnet buffers: %s", cudaGetErrorString(e));
	}

	int s = bnufft_precnet_set_params(n, params, stream);

	if (BNUFFT_OK != s) {

		bnufft_precnet_free(n);
		return s;
	}

	*out = n;
	return BNUFFT_OK;
}

extern "C" int bnufft_precnet_forward(bnufft_precnet_t n, void* out, const void* in, long X, long Y, long nimg, void* stream)
{
	cudaStream_t st = S(stream);

	if (!n || (X < 1) || (Y < 1) || (nimg < 1) || (X > (1 << 20)) || (Y > 65535 * NET_TILE_Y) || (nimg > 65535))
		return fail(BNUFFT_ERR_ARG, "bad precnet image size");

	const long P = X * Y * nimg;
	dim3 grid = net_tiles((int)X, (int)Y, nimg);
	TRY(net_ensure_ws(n, P, (long)grid.x * grid.y * grid.z));
	size_t b = sizeof(float2) * P;
	Staged i, o;
	TRY(stage_in(i, in, b, st));
	TRY(stage_out_alloc(o, out, b, st));
	TRY(net_forward(n, (const float2*)i.dev, (int)X, (int)Y, nimg, n->act, nullptr, nullptr, nullptr, 0, nullptr,
			(float2*)o.dev, nullptr, nullptr, nullptr, nullptr, nullptr, st));
	return stage_out_copy(o, out, b, st);
}

static int net_train(bnufft_precnet_t n, const void* in, const void* target, const void* gout_in, long X, long Y,
		long nimg, float lr, double* loss, float* grads, cudaStream_t st);

extern "C" int bnufft_precnet_train_step(bnufft_precnet_t n, const void* in, const void* target, long X, long Y,
		long nimg, float lr, double* loss, float* grads, void* stream)
{
	return net_train(n, in, target, nullptr, X, Y, nimg, lr, loss, grads, S(stream));
}

extern "C" int bnufft_precnet_backward(bnufft_precnet_t n, const void* in, const void* gout, long X, long Y,
		long nimg, float lr, float* grads, void* stream)
{
	return net_train(n, in, nullptr, gout, X, Y, nimg, lr, nullptr, grads, S(stream));
}

// forward with all activations, then the gradient of the loss (MSE against
// target) or the given output gradient gout_in, backward, optional Adam step
static int net_train(bnufft_precnet_t n, const void* in, const void* target, const void* gout_in, long X, long Y,
		long nimg, float lr, double* loss, float* grads, cudaStream_t st)
{

	if (!n || (X < 1) || (Y < 1) || (nimg < 1) || (X > (1 << 20)) || (Y > 65535 * NET_TILE_Y) || (nimg > 65535))
		return fail(BNUFFT_ERR_ARG, "bad precnet image size");

	const long P = X * Y * nimg;
	const int x = (int)X, y = (int)Y;
	dim3 grid = net_tiles(x, y, nimg);
	TRY(net_ensure_ws(n, P, (long)grid.x * grid.y * grid.z));
	size_t b = sizeof(float2) * P;
	Staged si, stg;
	TRY(stage_in(si, in, b, st));
	TRY(stage_in(stg, target ? target : gout_in, b, st));
	const float2* inp = (const float2*)si.dev;
	const unsigned pb = (unsigned)((P + NET_THREADS - 1) / NET_THREADS);

	// forward, keeping every layer's activation
	TRY(net_forward(n, inp, x, y, nimg, n->act, nullptr, nullptr, nullptr, 0, nullptr, n->out, nullptr, nullptr, nullptr,
			nullptr, nullptr, st));

	// loss = (1 / nimg) sum |out - target|^2, gout = dloss / dout
	if (target) {

		k_net_loss<<<NET_LOSS_BLOCKS, 256, 0, st>>>(n->out, (const float2*)stg.dev, P, 2.f / (float)nimg, n->gout, n->loss_part);
		LAUNCHED();

	} else {

		CUDA_TRY(cudaMemcpyAsync(n->gout, stg.dev, b, cudaMemcpyDeviceToDevice, st));
		loss = nullptr;
	}

	// backward: layer 6, then 5..2 on the tensor cores, then layer 1
	TRY((net_wgrad<NET_C, 2, bf16, float>(n, 5, n->act[4], (const float*)n->gout, x, y, nimg, st)));
	k_net_out_bwd<<<pb, NET_THREADS, 0, st>>>(n->gout, n->act[4], x, y, P, n->pr + NetLayout::woff(5), n->gu0);
	LAUNCHED();
	bf16* gu = n->gu0;
	bf16* gn = n->gu1;

	for (int l = 4; l >= 1; l--) {

		TRY((net_wgrad<NET_C, NET_C, bf16, bf16>(n, l, n->act[l - 1], gu, x, y, nimg, st)));
		TRY(launch_conv32<1>(n, gu, n->wt + (l - 1) * 9216, n->wt_tc + (l - 1) * 9216, nullptr, n->act[l - 1], gn, x,
				y, nimg, nullptr, nullptr, st));
		std::swap(gu, gn);
	}

	TRY((net_wgrad<2, NET_C, float, bf16>(n, 0, (const float*)inp, gu, x, y, nimg, st)));

	if (grads)
		CUDA_TRY(cudaMemcpyAsync(grads, n->grad, sizeof(float) * NET_N, cudaMemcpyDefault, st));

	if (lr > 0.f) {

		n->step++;
		const float b1 = 0.9f, b2 = 0.999f;
		float c1 = (float)(1. / (1. - pow((double)b1, n->step)));
		float c2 = (float)(1. / (1. - pow((double)b2, n->step)));
		k_adam<<<(NET_N + 255) / 256, 256, 0, st>>>(n->params, n->grad, n->m, n->v, NET_N, lr, b1, b2, 1e-8f, c1, c2);
		LAUNCHED();
		TRY(net_pack(n, st));
	}

	if (loss) {

		CUDA_TRY(cudaMemcpyAsync(n->loss_host, n->loss_part, sizeof(double) * NET_LOSS_BLOCKS, cudaMemcpyDeviceToHost, st));
		CUDA_TRY(cudaStreamSynchronize(st));
		double acc = 0.;

		for (int i = 0; i < NET_LOSS_BLOCKS; i++)
			acc += n->loss_host[i];

		*loss = acc / (double)nimg;
	}

	return BNUFFT_OK;
}

struct bnufft_pics_s {

	bnufft_plan_t nufft;
	bnufft_pics_conf conf;
	long C, npix, M;
	int cpg, groups;
	float2* sens = nullptr;		// [npix, C]
	float2* part = nullptr;		// [npix, groups] coil-sum partials
	float2 *x = nullptr, *r = nullptr, *b = nullptr;
	float2* pbuf[2] = { nullptr, nullptr };	// search direction, alternating by iteration
	float2* kbuf = nullptr;		// [M, C] (non-Toeplitz normal)
	float* mag = nullptr;		// [npix] |adj|
	SelectState* sel = nullptr;	// radix select of the scaling's order statistics
	double* pap_part = nullptr;	// p^H partial, one per final row-pass block
	double* pp_part = nullptr;	// ||p||^2, one per first row-pass block
	double* rs_part = nullptr;	// ||r||^2, one per CG step block
	// flexible CG (conf.precond): z = M(r); the last directions and their A p
	float2* z = nullptr;
	float2 *p_ring = nullptr, *ap_ring = nullptr;	// [FCG_RING][npix]
	double* dots_part = nullptr;	// <z, A p_j> partials [FCG_MAX_M][nparts]
	double* pr_part = nullptr;	// <p, r>, one per direction-update block
	int fcg_m = 1;			// truncation: directions orthogonalised against
	int ndots = 0;			// preconditioner last-pass blocks (folded <z, A p> partials)
	bool fcg_fold = true;		// fold the dot and test launches (BNUFFT_FCG_FOLD=0: not)
	bool fcg_fused = false;		// folded, and the direction update runs in the cluster
					// preconditioner (BNUFFT_FCG_FUSE=0: not)
	int ndir = 0;			// its <p, r> and ||p||^2 partials per launch
	bnufft_precnet_t net = nullptr;	// learned correction (conf.precond == 2), not owned
	float2* pinv_pad = nullptr;	// padded-circulant spectrum (conf.precond == 3), Toeplitz grid
	double* mcn_part = nullptr;	// ||M_circ(r)||^2 partials
	bf16* nact[2] = { nullptr, nullptr };	// its activations, ping-pong [npix][32]
	long max_row_blocks;
	int nparts;
	CgScalars* scal = nullptr;
	// the CG iterations as one graph: a while node whose body is one iteration
	cudaGraph_t cg_graph = nullptr;
	cudaGraph_t cg_body = nullptr;
	cudaGraphConditionalHandle cg_loop = 0;
	cudaGraphExec_t cg_exec = nullptr;
	int cg_dev = -1;
	int body_kernels = 0;
	long last_host_kernels = 0;	// launched from the host by the last run
	bool last_graph = false;	// last run's CG loop ran as the graph
	cudaEvent_t run_done = nullptr;	// recorded after each run on its stream
};

// The CG loop graph of a model (a while node whose body is one iteration)
// and, once its model is freed, the event of its last launch.
struct LoopGraph {

	int dev;
	cudaGraph_t graph;
	cudaGraph_t body;
	cudaGraphConditionalHandle loop;
	cudaGraphExec_t exec;
	cudaEvent_t done;
};

// Loop graphs of freed models, for reuse. Instantiating and destroying an
// executable per model costs the host hundreds of microseconds, and
// destroying one whose launch still runs can wait for the device. A new model
// instead clears a pooled graph's body, captures its own iteration into it
// (same graph, same conditional handle) and updates the executable in place
// (cudaGraphExecUpdate); an update applies to later launches only, so the
// freed model's last solve may still be running. When the topology differs
// (another solver or size) the update fails and the model instantiates its
// own graph.
enum { LOOP_POOL_MAX = 8 };
static std::mutex g_loop_mutex;
static std::vector<LoopGraph> g_loop_pool;

// Loop graphs that could not be reused, destroyed once their last launch has
// completed (checked without waiting on every create and free).
struct GraphGrave {

	cudaEvent_t done;
	cudaGraphExec_t exec;
	cudaGraph_t graph;
};

static std::mutex g_grave_mutex;
static std::vector<GraphGrave> g_grave;

static void bury(const LoopGraph& lg)
{
	std::lock_guard<std::mutex> lock(g_grave_mutex);
	g_grave.push_back(GraphGrave{ lg.done, lg.exec, lg.graph });
}

static void reap_graves()
{
	std::lock_guard<std::mutex> lock(g_grave_mutex);
	size_t k = 0;

	for (size_t i = 0; i < g_grave.size(); i++) {

		GraphGrave& g = g_grave[i];
		cudaError_t e = cudaEventQuery(g.done);

		if (cudaErrorNotReady == e) {

			cudaGetLastError();	// not an error: clear it
			g_grave[k++] = g;
			continue;
		}

		cudaGraphExecDestroy(g.exec);

		if (g.graph)
			cudaGraphDestroy(g.graph);

		cudaEventDestroy(g.done);
	}

	g_grave.resize(k);
}

extern "C" void bnufft_pics_conf_defaults(struct bnufft_pics_conf* c)
{
	c->lambda = 0.f;
	c->maxiter = 30;
	c->tol = 0.f;
	c->scaling = 0.f;
	c->rescale = 0;
	c->toeplitz = 1;
	c->periodic = 0;
	c->deterministic = 0;
	c->bin = 0;
	c->precond = 0;
	c->ref_scalars = 1;
	c->net_iters = 1;
}

// A^H A x (+ lam x), with optional per-block Re<x, out> partials
static int sense_normal(bnufft_pics_s* ps, const float2* x, float2* out, float lam, double* dot_part,
		const int* done, cudaStream_t st)
{
	OpCtx& op = ps->nufft->op;

	if (ps->nufft->psf) {

		TRY(op_toeplitz(toe_ctx(ps->nufft), toe_psf(ps->nufft, st), x, ps->sens, ps->C, ps->cpg, ps->part, st));

	} else {

		TRY(op_forward(op, x, ps->sens, ps->C, ps->kbuf, st));
		TRY(op_adjoint(op, ps->kbuf, ps->sens, ps->C, ps->cpg, ps->part, st));
	}

	k_combine<<<ps->nparts, RED_THREADS, 0, st>>>(out, ps->part, ps->groups, ps->npix, x, lam, dot_part, done);
	LAUNCHED();
	return BNUFFT_OK;
}

static int build_precond_pad(bnufft_pics_s* ps, cudaStream_t st);

extern "C" int bnufft_pics_create(bnufft_pics_t* out, int N, const long ksp_dims[], const long sens_dims[],
		const long traj_dims[], const void* traj, const void* sens,
		const struct bnufft_pics_conf* conf_in, void* stream)
{
	*out = nullptr;
	cudaStream_t st = S(stream);
	bnufft_pics_conf conf;
	reap_graves();

	if (conf_in)
		conf = *conf_in;
	else
		bnufft_pics_conf_defaults(&conf);

	if (N < 5)
		return fail(BNUFFT_ERR_ARG, "need N >= 5 dims");

	for (int i = 4; i < N; i++)
		if ((1 != ksp_dims[i]) || (1 != sens_dims[i]))
			return fail(BNUFFT_ERR_UNSUPPORTED, "dim %d must be 1 (one set of maps, one image)", i);

	if (ksp_dims[3] != sens_dims[3])
		return fail(BNUFFT_ERR_ARG, "coil dims differ (%ld, %ld)", ksp_dims[3], sens_dims[3]);

	if (conf.maxiter < 0)
		return fail(BNUFFT_ERR_ARG, "maxiter < 0");

	bnufft_conf nc;
	bnufft_conf_defaults(&nc);
	nc.toeplitz = conf.toeplitz;
	nc.periodic = conf.periodic;
	nc.deterministic = conf.deterministic;
	nc.bin = conf.bin;

	if ((conf.precond < 0) || (conf.precond > 3))
		return fail(BNUFFT_ERR_ARG, "precond must be 0, 1, 2 or 3");

	if (conf.precond && !conf.toeplitz)
		return fail(BNUFFT_ERR_UNSUPPORTED, "the circulant preconditioner needs the Toeplitz normal operator");

	auto ps = new bnufft_pics_s();
	ps->conf = conf;
	int s = bnufft_create2(&ps->nufft, N, ksp_dims, sens_dims, traj_dims, traj, nullptr, nullptr, nullptr, nullptr, &nc, stream);

	if (BNUFFT_OK != s) {

		delete ps;
		return s;
	}

	ps->C = sens_dims[3];
	ps->npix = ps->nufft->op.g.npix;
	ps->M = ps->nufft->op.g.M;

	// coil groups of the coil-summing row pass: the fewest coils per block
	// whose blocks all fit one wave of resident blocks (two per SM), so no
	// partial second wave idles the SMs, and fewer partials to combine
	// (256^2, 16 coils: 2 coils per block, 3.6% faster solve than 1)
	long YZ = (long)ps->nufft->op.g.N[1] * ps->nufft->op.g.N[2];
	int Brow = choose_B(ps->nufft->op.g.G[0], YZ * ps->C);
	long rowblocks = (YZ + Brow - 1) / Brow;
	const long slots = 2 * 148;
	ps->cpg = (int)std::max<long>(1, std::min<long>(ps->C, (rowblocks * ps->C + slots - 1) / slots));
	ps->groups = (int)((ps->C + ps->cpg - 1) / ps->cpg);
	ps->nparts = (int)vec_blocks(ps->npix);

	auto ck = [&](cudaError_t e) { if (cudaSuccess != e && BNUFFT_OK == s) s = fail(BNUFFT_ERR_NOMEM, "pics buffers: %s", cudaGetErrorString(e)); };
	// maps from the host are copied on the copy stream: allocated in its order
	cudaStream_t mst = on_device(sens) ? st : copy_stream();
	ck(cudaMallocAsync(&ps->sens, sizeof(float2) * ps->npix * ps->C, mst ? mst : st));
	ck(cudaMallocAsync(&ps->part, sizeof(float2) * ps->npix * ps->groups, st));
	ck(cudaMallocAsync(&ps->x, sizeof(float2) * ps->npix, st));
	ck(cudaMallocAsync(&ps->r, sizeof(float2) * ps->npix, st));
	ck(cudaMallocAsync(&ps->pbuf[0], sizeof(float2) * ps->npix, st));
	ck(cudaMallocAsync(&ps->pbuf[1], sizeof(float2) * ps->npix, st));
	ck(cudaMallocAsync(&ps->b, sizeof(float2) * ps->npix, st));
	ck(cudaMallocAsync(&ps->mag, sizeof(float) * ps->npix, st));
	ck(cudaMallocAsync(&ps->sel, sizeof(SelectState), st));

	if (ps->sel)
		ck(cudaMemsetAsync(ps->sel, 0, sizeof(SelectState), st));
	// row-pass blocks hold at least 4 rows: bounds for the partial arrays
	ps->max_row_blocks = (YZ + 3) / 4 * ps->C + 1;
	ck(cudaMallocAsync(&ps->pap_part, sizeof(double) * ps->max_row_blocks, st));
	// ||p||^2 partials: per first row-pass block (plain CG) or per vector block (flexible CG)
	ck(cudaMallocAsync(&ps->pp_part, sizeof(double) * std::max<long>(ps->max_row_blocks, ps->nparts), st));
	ck(cudaMallocAsync(&ps->rs_part, sizeof(double) * ps->nparts, st));
	ck(cudaMallocAsync(&ps->scal, sizeof(CgScalars), st));

	if (!conf.toeplitz)
		ck(cudaMallocAsync(&ps->kbuf, sizeof(float2) * ps->M * ps->C, st));

	if (conf.precond) {

		// the circulant preconditioners are linear (flexible CG keeps one
		// direction, as PCG); the learned one is not: keep FCG_MAX_M, or
		// one direction when it is used in the first iterations only
		ps->fcg_m = ((2 == conf.precond) && (conf.net_iters <= 0)) ? (int)FCG_MAX_M : 1;

		if (const char* e = getenv("BNUFFT_FCG_M"))
			ps->fcg_m = std::max(1, std::min((int)FCG_MAX_M, atoi(e)));

		if (const char* e = getenv("BNUFFT_FCG_FOLD"))
			ps->fcg_fold = (0 != strcmp(e, "0"));

		ck(cudaMallocAsync(&ps->z, sizeof(float2) * ps->npix, st));
		ck(cudaMallocAsync(&ps->p_ring, sizeof(float2) * ps->npix * FCG_RING, st));
		ck(cudaMallocAsync(&ps->ap_ring, sizeof(float2) * ps->npix * FCG_RING, st));
		ck(cudaMallocAsync(&ps->dots_part, sizeof(double) * std::max<long>((long)ps->nparts * FCG_MAX_M,
				ps->max_row_blocks), st));
		ck(cudaMallocAsync(&ps->pr_part, sizeof(double) * ps->nparts, st));

		if (BNUFFT_OK == s) {	// after the PSF, on the stream that builds it

			int dev = 0;
			const AuxStream* aux = (ps->nufft->psf_ev && (cudaSuccess == cudaGetDevice(&dev))) ? aux_stream(dev) : nullptr;
			cudaStream_t pst = aux ? aux->st : st;

			if ((2 == conf.precond) || (3 == conf.precond))
				s = build_precond_pad(ps, pst);
			else
				s = build_precond(ps->nufft, pst);

			if (ps->nufft->psf_ev)
				cudaEventRecord(ps->nufft->psf_ev, pst);
		}
	}

	if (BNUFFT_OK == s) {

		const size_t mb = sizeof(float2) * ps->npix * ps->C;

		if (on_device(sens)) {

			cudaError_t e = cudaMemcpyAsync(ps->sens, sens, mb, cudaMemcpyDeviceToDevice, st);

			if (cudaSuccess != e)
				s = fail(BNUFFT_ERR_CUDA, "maps upload: %s", cudaGetErrorString(e));

		} else {	// returns once the host array has been read

			s = copy_in(ps->sens, sens, mb, st);
		}
	}

	if (BNUFFT_OK != s) {

		std::string msg = g_err;
		bnufft_pics_free(ps);
		g_err = msg;
		return s;
	}

	*out = ps;
	return BNUFFT_OK;
}

extern "C" int bnufft_pics_normal(bnufft_pics_t ps, void* dst, const void* src, void* stream)
{
	cudaStream_t st = S(stream);
	size_t b = sizeof(float2) * ps->npix;
	Staged i, o;
	TRY(stage_in(i, src, b, st));
	TRY(stage_out_alloc(o, dst, b, st));
	TRY(sense_normal(ps, (const float2*)i.dev, (float2*)o.dev, 0.f, nullptr, nullptr, st));
	return stage_out_copy(o, dst, b, st);
}

// b = A^H y / scale into ps->b: adjoint (coil-sum partials, then combine) and
// the data scaling of src/pics.c:499-530 (y /= scale  <=>  A^H y /= scale)
static int pics_prologue(bnufft_pics_s* ps, const float2* ksp, cudaStream_t st)
{
	OpCtx& op = ps->nufft->op;
	unsigned nb = (unsigned)ps->nparts;
	TRY(op_adjoint(op, ksp, ps->sens, ps->C, ps->cpg, ps->part, st));
	k_combine<<<nb, RED_THREADS, 0, st>>>(ps->b, ps->part, ps->groups, ps->npix, nullptr, 0.f, nullptr, nullptr);
	LAUNCHED();

	if (0.f == ps->conf.scaling) {

		// three order statistics of |b| by radix select (estimate_scaling_norm)
		const unsigned sb = (unsigned)std::max(1L, std::min<long>((ps->npix + 4 * SEL_THREADS - 1) / (4 * SEL_THREADS), 2 * 148));
		k_select_pass<0><<<sb, SEL_THREADS, 0, st>>>(ps->b, ps->mag, ps->npix, ps->sel, ps->scal);
		LAUNCHED();
		k_select_pass<1><<<sb, SEL_THREADS, 0, st>>>(ps->b, ps->mag, ps->npix, ps->sel, ps->scal);
		LAUNCHED();
		k_select_pass<2><<<sb, SEL_THREADS, 0, st>>>(ps->b, ps->mag, ps->npix, ps->sel, ps->scal);
		LAUNCHED();

	} else {

		k_set_scaling<<<1, 1, 0, st>>>(ps->scal, ps->conf.scaling);
		LAUNCHED();
	}

	k_scale_dev<<<nb, RED_THREADS, 0, st>>>(ps->b, ps->b, ps->npix, &ps->scal->inv_scale);
	LAUNCHED();
	return BNUFFT_OK;
}

// One CG iteration on (A^H A + lambda) x = b in four passes: the direction
// update fused into the first row pass, the normal operator's column passes,
// the final row pass with the p^H A p partials, and the x / r step with the
// ||r||^2 partials. it < 0: the kernels take the iteration index from the
// device counter (the loop runs inside a graph).
static int pics_iteration(bnufft_pics_s* ps, int it, cudaStream_t st)
{
	bool toep = (nullptr != ps->nufft->psf);
	OpCtx& op = toep ? toe_ctx(ps->nufft) : ps->nufft->op;	// Toeplitz: its (embedding) grid
	const Geom& g = op.g;
	long YZ = (long)g.N[1] * g.N[2];
	const int* done = &ps->scal->done;
	float2* p_prev = ps->pbuf[0];
	float2* p_cur = ps->pbuf[1];
	int npp = 0, npap = 0;

	TRY(rows_fwd_cg(g.G[0], ps->b, ps->r, p_prev, p_cur, ps->sens, toep ? nullptr : op.ax, op.ayz,
			g.N[0], YZ, YZ * ps->C, op.w.t1, ps->scal, it, ps->rs_part, ps->nparts, ps->pp_part, &npp, st));

	DotHook dh;
	dh.p = p_cur;
	dh.part = ps->pap_part;
	dh.done = done;
	dh.nblocks = &npap;

	if (toep) {

		TRY(op_toeplitz_cols(op, toe_psf(ps->nufft, st), ps->C, st, done));
		TRY(rows_inv(g.G[0], op.w.t1, ps->sens, nullptr, nullptr, g.N[0], YZ, (int)ps->C, ps->cpg, ps->part, st,
				dh.p, dh.part, dh.done, dh.nblocks));

	} else {

		TRY(op_spectrum_cols(op, ps->C, op.w.grid, st));
		TRY(degrid(op, op.w.grid, ps->C, ps->kbuf, st));
		TRY(op_adjoint(op, ps->kbuf, ps->sens, ps->C, ps->cpg, ps->part, st, dh));
	}

	if ((npp > ps->max_row_blocks) || (npap > ps->max_row_blocks))
		return fail(BNUFFT_ERR_ARG, "internal: partial arrays too small");

	k_cg_step<<<(unsigned)ps->nparts, RED_THREADS, 0, st>>>(ps->x, ps->r, p_cur, ps->part, ps->groups, ps->npix,
			ps->conf.lambda, ps->scal, it, ps->pap_part, npap, ps->pp_part, npp, ps->rs_part, p_prev);
	LAUNCHED();
	return BNUFFT_OK;
}

static int pics_precond_circ(bnufft_pics_s* ps, const float2* r, float2* z, const float2* pdot, double* dot_part,
		int* nblocks, cudaStream_t st, const PcDir* dir = nullptr);

// the padded-circulant spectrum 1/(|P| + mu) on the Toeplitz grid (precond 3,
// k_precond_pad_spectrum), built after the PSF on the stream that builds it
static int build_precond_pad(bnufft_pics_s* ps, cudaStream_t st)
{
	bnufft_plan_s* p = ps->nufft;

	if (!p->psf)
		return fail(BNUFFT_ERR_ARG, "the padded preconditioner needs the Toeplitz PSF");

	const Geom& g = toe_ctx(p).g;
	const float mu_lam = (float)(2.5 * ps->conf.lambda * std::pow(4., (double)g.nd) / (double)g.gsz);
	CUDA_TRY(cudaMallocAsync(&ps->pinv_pad, sizeof(float2) * g.gsz, st));
	k_precond_pad_spectrum<<<vec_blocks(g.gsz), RED_THREADS, 0, st>>>(ps->pinv_pad, toe_psf(p, st), g.gsz, mu_lam);
	LAUNCHED();
	return BNUFFT_OK;
}

// z = crop F^-1 (|P| + mu)^-1 F pad r: the Toeplitz passes on one image with
// the padded-circulant spectrum in place of the PSF (the plan's buffers,
// free between the normal operator's passes); optional partials Re<pdot, z>
static int pics_precond_pad(bnufft_pics_s* ps, const float2* r, float2* z, const float2* pdot, double* dot_part,
		int* nblocks, cudaStream_t st)
{
	bnufft_plan_s* p = ps->nufft;
	OpCtx& op = toe_ctx(p);
	const Geom& g = op.g;
	const int* done = &ps->scal->done;
	long YZ = (long)g.N[1] * g.N[2];
	psf_wait(p, st);
	TRY(alloc_work(op.w, g, 1, st));	// allocates only outside a solve (which sizes it first)
	t_prof_precond = true;
	int s = rows_fwd(g.G[0], r, nullptr, nullptr, nullptr, g.N[0], YZ, YZ, op.w.t1, st, done);

	if (BNUFFT_OK == s)
		s = op_toeplitz_cols(op, ps->pinv_pad, 1, st, done);

	if (BNUFFT_OK == s)
		s = rows_inv(g.G[0], op.w.t1, nullptr, nullptr, nullptr, g.N[0], YZ, 1, 1, z, st, pdot, dot_part, done, nblocks);

	t_prof_precond = false;
	return s;
}

// z = M(r): the circulant preconditioner (precond 1), the padded one
// (precond 3), or the padded one plus the learned correction
// ||M_pad(r)|| net(M_pad(r) / ||M_pad(r)||) (precond 2; the norm from the
// partials of the pass that wrote M_pad(r)); optional partials Re<pdot, z>
static int pics_precond(bnufft_pics_s* ps, const float2* r, float2* z, const float2* pdot, double* dot_part,
		int* nblocks, cudaStream_t st)
{
	if (3 == ps->conf.precond)
		return pics_precond_pad(ps, r, z, pdot, dot_part, nblocks, st);

	if (2 != ps->conf.precond)
		return pics_precond_circ(ps, r, z, pdot, dot_part, nblocks, st);

	if (!ps->net)
		return fail(BNUFFT_ERR_ARG, "precond 2 needs a network (bnufft_pics_set_precnet)");

	// z = M_pad(r) with the partials of ||z||^2, then z += ||z|| net(z / ||z||):
	// flexible CG is invariant to a positive scale of z per iteration, so the
	// network learns a scale-free correction of the padded-circulant step
	// from the step itself
	int nmc = 0;
	TRY(pics_precond_pad(ps, r, z, z, ps->mcn_part, &nmc, st));

	if (nmc > ps->max_row_blocks)
		return fail(BNUFFT_ERR_ARG, "internal: partial arrays too small");

	const Geom& g = ps->nufft->op.g;
	bf16* acts[5] = { ps->nact[0], ps->nact[1], ps->nact[0], ps->nact[1], ps->nact[0] };
	CgScalars* sc = ps->scal;
	return net_forward(ps->net, z, g.N[0], g.N[1], 1, acts, nullptr, nullptr, ps->mcn_part, nmc, z, z, pdot,
			dot_part, nblocks, &sc->done, &sc->net_off, st, ps->mcn_part, nmc);
}

// the one-launch cluster form of the circulant preconditioner (square 2D
// images of 64, 128 or 256 pixels a side; BNUFFT_PRECOND_CLUSTER=0: the
// three-pass form): one cluster of CL CTAs
template <int N, int CL>
static int launch_precond_cluster(const float2* r, const float2* pinv, float2* z, const float2* pdot,
		double* dot_part, const int* done, const PcDir& dir, cudaStream_t st)
{
	using Sh = PrecondClusterShape<N, CL>;
	const float2* tw;
	TRY(get_twiddles(N, &tw));
	cudaLaunchConfig_t cfg = {};
	cudaLaunchAttribute at[1];
	at[0].id = cudaLaunchAttributeClusterDimension;
	at[0].val.clusterDim.x = CL;
	at[0].val.clusterDim.y = 1;
	at[0].val.clusterDim.z = 1;
	cfg.gridDim = dim3(CL);
	cfg.blockDim = dim3(Sh::NT);
	cfg.dynamicSmemBytes = Sh::SMEM;
	cfg.stream = st;
	cfg.attrs = at;
	cfg.numAttrs = 1;
	cudaEvent_t pe = prof_begin("cluster", st);
	cudaError_t e = cudaLaunchKernelEx(&cfg, k_precond_cluster<N, CL>, r, pinv, z, tw, pdot, dot_part, done, dir);
	prof_end(pe, st);
	g_launches.fetch_add(1, std::memory_order_relaxed);

	if (cudaSuccess != e)
		return fail(BNUFFT_ERR_CUDA, "preconditioner cluster launch: %s", cudaGetErrorString(e));

	return BNUFFT_OK;
}

// whether one cluster of CL CTAs with their shared memory fits this device
// (16 is a non-portable cluster size), once per size and device
template <int N, int CL>
static bool precond_cluster_fits()
{
	static std::mutex m;
	static std::map<int, bool> fits;
	int dev = 0;

	if (cudaSuccess != cudaGetDevice(&dev))
		return false;

	std::lock_guard<std::mutex> lock(m);
	auto it = fits.find(dev);

	if (it != fits.end())
		return it->second;

	using Sh = PrecondClusterShape<N, CL>;
	auto kern = k_precond_cluster<N, CL>;
	bool ok = (cudaSuccess == cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::SMEM));

	if (ok && (CL > 8))
		ok = (cudaSuccess == cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));

	if (ok) {

		cudaLaunchConfig_t cfg = {};
		cudaLaunchAttribute at[1];
		at[0].id = cudaLaunchAttributeClusterDimension;
		at[0].val.clusterDim.x = CL;
		at[0].val.clusterDim.y = 1;
		at[0].val.clusterDim.z = 1;
		cfg.gridDim = dim3(CL);
		cfg.blockDim = dim3(Sh::NT);
		cfg.dynamicSmemBytes = Sh::SMEM;
		cfg.attrs = at;
		cfg.numAttrs = 1;
		int nc = 0;
		ok = (cudaSuccess == cudaOccupancyMaxActiveClusters(&nc, kern, &cfg)) && (nc > 0);
	}

	cudaGetLastError();
	fits[dev] = ok;
	return ok;
}

// the cluster size for this image (0: use the three-pass form)
static int precond_cluster_size(const Geom& g)
{
	if (const char* e = getenv("BNUFFT_PRECOND_CLUSTER"))
		if (0 == strcmp(e, "0"))
			return 0;

	if ((1 != g.N[2]) || (g.N[0] != g.N[1]))
		return 0;

	switch (g.N[0]) {
	case 64: return precond_cluster_fits<64, 16>() ? 16 : (precond_cluster_fits<64, 8>() ? 8 : 0);
	case 128: return precond_cluster_fits<128, 16>() ? 16 : (precond_cluster_fits<128, 8>() ? 8 : 0);
	case 256: return precond_cluster_fits<256, 16>() ? 16 : (precond_cluster_fits<256, 8>() ? 8 : 0);
	default: return 0;
	}
}

// the circulant preconditioner applied to one image (N-point transforms, no
// padding)
// dir: the flexible-CG direction update fused into the cluster form (only
// where precond_cluster_size is nonzero)
static int pics_precond_circ(bnufft_pics_s* ps, const float2* r, float2* z, const float2* pdot, double* dot_part,
		int* nblocks, cudaStream_t st, const PcDir* dir)
{
	bnufft_plan_s* p = ps->nufft;
	const int* done = &ps->scal->done;
	PcDir nodir = {};
	const PcDir& d = dir ? *dir : nodir;

	if (const int cl = precond_cluster_size(p->op.g)) {

		int s = BNUFFT_OK;
		const int n = p->op.g.N[0];
		t_prof_precond = true;

		if (16 == cl)
			s = (64 == n) ? launch_precond_cluster<64, 16>(r, precond_spec(p, st), z, pdot, dot_part, done, d, st)
				: (128 == n) ? launch_precond_cluster<128, 16>(r, precond_spec(p, st), z, pdot, dot_part, done, d, st)
				: launch_precond_cluster<256, 16>(r, precond_spec(p, st), z, pdot, dot_part, done, d, st);
		else
			s = (64 == n) ? launch_precond_cluster<64, 8>(r, precond_spec(p, st), z, pdot, dot_part, done, d, st)
				: (128 == n) ? launch_precond_cluster<128, 8>(r, precond_spec(p, st), z, pdot, dot_part, done, d, st)
				: launch_precond_cluster<256, 8>(r, precond_spec(p, st), z, pdot, dot_part, done, d, st);

		t_prof_precond = false;

		if (nblocks)
			*nblocks = cl;

		return s;
	}

	if (dir)
		return fail(BNUFFT_ERR_ARG, "internal: fused direction without the cluster preconditioner");
	OpCtx full;
	full.g = p->op.g;

	for (int a = 0; a < 3; a++)
		full.g.G[a] = full.g.N[a];

	full.g.gsz = full.g.npix;
	full.kb = p->op.kb;
	full.traj = nullptr;
	full.w = p->op.w;	// the plan's buffers (N <= 2N), free between the operator's passes
	const Geom& g = full.g;
	long YZ = (long)g.N[1] * g.N[2];
	t_prof_precond = true;
	int s = rows_fwd(g.G[0], r, nullptr, nullptr, nullptr, g.N[0], YZ, YZ, full.w.t1, st, done);

	if (BNUFFT_OK == s)
		s = op_toeplitz_cols(full, precond_spec(p, st), 1, st, done);

	if (BNUFFT_OK == s)
		s = rows_inv(g.G[0], full.w.t1, nullptr, nullptr, nullptr, g.N[0], YZ, 1, 1, z, st, pdot, dot_part, done, nblocks);

	t_prof_precond = false;
	return s;
}

// One flexible-CG iteration: <z, A p_j> over the kept directions, the
// direction update, the normal operator's passes (as in plain CG), the step,
// the convergence test and z = M(r) for the next iteration. With the linear
// circulant preconditioner and one kept direction (the default of precond
// 1) two launches are folded away: <z, A p> comes from the preconditioner's
// last pass and the convergence test runs in the next direction update.
static int pics_fcg_iteration(bnufft_pics_s* ps, int it, cudaStream_t st)
{
	OpCtx& op = toe_ctx(ps->nufft);
	const Geom& g = op.g;
	long YZ = (long)g.N[1] * g.N[2];
	const int* done = &ps->scal->done;
	float2* p = ps->pbuf[1];
	unsigned nb = (unsigned)ps->nparts;
	int npap = 0;
	const bool folded = (1 == ps->fcg_m) && ps->fcg_fold;
	const int ring = (1 == ps->fcg_m) ? 1 : (int)FCG_RING;

	if (folded && ps->fcg_fused) {	// five launches: the normal's passes, the step, the
					// cluster preconditioner with the next direction
		TRY(rows_fwd(g.G[0], p, ps->sens, nullptr, nullptr, g.N[0], YZ, YZ * ps->C, op.w.t1, st, done));
		TRY(op_toeplitz_cols(op, toe_psf(ps->nufft, st), ps->C, st, done));
		TRY(rows_inv(g.G[0], op.w.t1, ps->sens, nullptr, nullptr, g.N[0], YZ, (int)ps->C, ps->cpg, ps->part, st,
				p, ps->pap_part, done, &npap));

		if (npap > ps->max_row_blocks)
			return fail(BNUFFT_ERR_ARG, "internal: partial arrays too small");

		k_fcg_step<<<nb, RED_THREADS, 0, st>>>(ps->x, ps->r, p, ps->ap_ring, 1, ps->part, ps->groups, ps->npix,
				ps->conf.lambda, ps->scal, it, ps->pap_part, npap, ps->pp_part, ps->ndir, ps->pr_part, ps->ndir,
				ps->rs_part);
		LAUNCHED();
		PcDir d = { ps->scal, it, 0, ps->rs_part, ps->nparts, p, ps->r, ps->pr_part, ps->pp_part };
		int nd = 0;
		TRY(pics_precond_circ(ps, ps->r, ps->z, ps->ap_ring, nullptr, &nd, st, &d));

		if (nd != ps->ndir)
			return fail(BNUFFT_ERR_ARG, "internal: preconditioner block count changed");

		return BNUFFT_OK;
	}

	if (!folded) {

		k_fcgm_dots<<<nb, RED_THREADS, 0, st>>>(ps->z, ps->ap_ring, ps->npix, ps->scal, it, ps->fcg_m, ring, ps->dots_part);
		LAUNCHED();
	}

	k_fcgm_dir<<<nb, RED_THREADS, 0, st>>>(p, ps->p_ring, ps->z, ps->r, ps->npix, ps->scal, it, ps->fcg_m, ring,
			ps->dots_part, folded ? ps->ndots : ps->nparts, ps->pr_part, ps->pp_part,
			folded ? ps->rs_part : nullptr, ps->nparts);
	LAUNCHED();
	TRY(rows_fwd(g.G[0], p, ps->sens, nullptr, nullptr, g.N[0], YZ, YZ * ps->C, op.w.t1, st, done));
	TRY(op_toeplitz_cols(op, toe_psf(ps->nufft, st), ps->C, st, done));
	TRY(rows_inv(g.G[0], op.w.t1, ps->sens, nullptr, nullptr, g.N[0], YZ, (int)ps->C, ps->cpg, ps->part, st,
			p, ps->pap_part, done, &npap));

	if (npap > ps->max_row_blocks)
		return fail(BNUFFT_ERR_ARG, "internal: partial arrays too small");

	k_fcg_step<<<nb, RED_THREADS, 0, st>>>(ps->x, ps->r, p, ps->ap_ring, ring, ps->part, ps->groups, ps->npix,
			ps->conf.lambda, ps->scal, it, ps->pap_part, npap, ps->pp_part, ps->nparts, ps->pr_part, ps->nparts,
			ps->rs_part);
	LAUNCHED();

	if (folded) {

		int nd = 0;
		TRY(pics_precond(ps, ps->r, ps->z, ps->ap_ring, ps->dots_part, &nd, st));

		if (nd != ps->ndots)
			return fail(BNUFFT_ERR_ARG, "internal: preconditioner block count changed");

		return BNUFFT_OK;
	}

	k_fcg_check<<<1, RED_THREADS, 0, st>>>(ps->scal, it, ps->rs_part, ps->nparts);
	LAUNCHED();
	return pics_precond(ps, ps->r, ps->z, nullptr, nullptr, nullptr, st);
}

static int pics_any_iteration(bnufft_pics_s* ps, int it, cudaStream_t st)
{
	return ps->conf.precond ? pics_fcg_iteration(ps, it, st) : pics_iteration(ps, it, st);
}

// per thread and device: the stream the loop graphs are captured on
static cudaStream_t capture_stream(int dev)
{
	static thread_local std::map<int, cudaStream_t> streams;
	auto it = streams.find(dev);

	if (it != streams.end())
		return it->second;

	cudaStream_t s = nullptr;

	if (cudaSuccess != cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking))
		return nullptr;

	streams[dev] = s;
	return s;
}

// one iteration and k_cg_advance, captured into the (empty) loop body
static int capture_body(bnufft_pics_s* ps, cudaStream_t cap, cudaGraph_t body, cudaGraphConditionalHandle loop)
{
	CUDA_TRY(cudaStreamBeginCaptureToGraph(cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
	long before = g_launches.load();
	int s = pics_any_iteration(ps, -1, cap);

	if (BNUFFT_OK == s) {

		k_cg_advance<<<1, 1, 0, cap>>>(ps->scal, loop);
		cudaError_t e = cudaGetLastError();

		if (cudaSuccess != e)
			s = fail(BNUFFT_ERR_CUDA, "loop capture: %s", cudaGetErrorString(e));

		g_launches.fetch_add(1);
	}

	// captured kernels are not launches: counted when the graph runs
	ps->body_kernels = (int)(g_launches.load() - before);
	g_launches.fetch_sub(ps->body_kernels);

	cudaGraph_t captured = nullptr;
	cudaError_t e = cudaStreamEndCapture(cap, &captured);

	if (BNUFFT_OK != s)
		return s;

	CUDA_TRY(e);
	return BNUFFT_OK;
}

// a pooled loop graph of this device updated to this model's iteration
static bool reuse_loop_graph(bnufft_pics_s* ps, cudaStream_t cap, int dev)
{
	LoopGraph lg;
	bool found = false;

	{
		std::lock_guard<std::mutex> lock(g_loop_mutex);

		for (size_t i = 0; i < g_loop_pool.size(); i++) {

			if (g_loop_pool[i].dev == dev) {

				lg = g_loop_pool[i];
				g_loop_pool.erase(g_loop_pool.begin() + i);
				found = true;
				break;
			}
		}
	}

	if (!found)
		return false;

	size_t n = 0;
	cudaError_t e = cudaGraphGetNodes(lg.body, nullptr, &n);
	std::vector<cudaGraphNode_t> nodes(n);

	if ((cudaSuccess == e) && (n > 0))
		e = cudaGraphGetNodes(lg.body, nodes.data(), &n);

	for (size_t i = 0; (cudaSuccess == e) && (i < n); i++)
		e = cudaGraphDestroyNode(nodes[i]);

	if ((cudaSuccess == e) && (BNUFFT_OK == capture_body(ps, cap, lg.body, lg.loop))) {

		cudaGraphExecUpdateResultInfo info;
		e = cudaGraphExecUpdate(lg.exec, lg.graph, &info);

		if (cudaSuccess == e) {

			ps->cg_graph = lg.graph;
			ps->cg_body = lg.body;
			ps->cg_loop = lg.loop;
			ps->cg_exec = lg.exec;
			ps->cg_dev = dev;
			cudaEventDestroy(lg.done);
			return true;
		}
	}

	// not reusable (the executable is unchanged): destroyed once idle
	cudaGetLastError();
	g_err.clear();
	bury(lg);
	return false;
}

// Capture the CG loop once: a graph holding one while node whose body is an
// iteration followed by k_cg_advance, which continues the loop until the
// solve converged or reached maxiter. One graph launch then runs the whole
// loop with no host round trip and no launches past convergence.
static int capture_cg_loop(bnufft_pics_s* ps)
{
	int dev;
	CUDA_TRY(cudaGetDevice(&dev));
	cudaStream_t cap = capture_stream(dev);

	if (!cap)
		return fail(BNUFFT_ERR_CUDA, "capture stream");

	if (reuse_loop_graph(ps, cap, dev))
		return BNUFFT_OK;

	CUDA_TRY(cudaGraphCreate(&ps->cg_graph, 0));
	CUDA_TRY(cudaGraphConditionalHandleCreate(&ps->cg_loop, ps->cg_graph, 1, cudaGraphCondAssignDefault));

	cudaGraphNodeParams np = {};
	np.type = cudaGraphNodeTypeConditional;
	np.conditional.handle = ps->cg_loop;
	np.conditional.type = cudaGraphCondTypeWhile;
	np.conditional.size = 1;
	cudaGraphNode_t node;
	CUDA_TRY(cudaGraphAddNode(&node, ps->cg_graph, nullptr, 0, &np));
	ps->cg_body = np.conditional.phGraph_out[0];
	ps->cg_dev = dev;
	TRY(capture_body(ps, cap, ps->cg_body, ps->cg_loop));
	CUDA_TRY(cudaGraphInstantiate(&ps->cg_exec, ps->cg_graph, 0));
	return BNUFFT_OK;
}

static bool cg_graph_enabled()
{
	// per-launch profiling needs the kernels launched one by one
	if (g_prof_active.load(std::memory_order_relaxed))
		return false;

	const char* e = getenv("BNUFFT_CG_GRAPH");
	return !(e && (0 == strcmp(e, "0")));
}

// One reconstruction from device k-space into a device image: data scaling,
// CG start, the iterations (as the while-node graph, or host-launched when
// graph is false, e.g. while the caller captures), the result.
static int pics_solve(bnufft_pics_s* ps, const float2* ksp, float2* out, cudaStream_t st, bool graph)
{
	OpCtx& op = ps->nufft->op;
	unsigned nb = (unsigned)ps->nparts;
	size_t ib = sizeof(float2) * ps->npix;
	ps->last_graph = false;
	TRY(pics_prologue(ps, ksp, st));

	// CG from zero (conjgrad, src/iter/italgos.c:497-572)
	k_cg_init<<<nb, RED_THREADS, 0, st>>>(ps->x, ps->r, ps->pbuf[1], ps->b, ps->npix, ps->rs_part);
	LAUNCHED();
	k_cg_start<<<1, RED_THREADS, 0, st>>>(ps->scal, ps->rs_part, ps->nparts, ps->conf.tol, ps->conf.maxiter,
			(0 == ps->conf.precond) && ps->conf.ref_scalars, (2 == ps->conf.precond) ? ps->conf.net_iters : 0);
	LAUNCHED();

	TRY(alloc_work(op.w, op.g, ps->C, st));

	if (ps->nufft->embed)
		TRY(alloc_work(ps->nufft->toe.w, ps->nufft->toe.g, ps->C, st));

	// the adjoint and the scaling above ran while the auxiliary stream built
	// the PSF (and the preconditioner); the iterations need them (the loop
	// graph's capture does not wait, so the stream waits here)
	psf_wait(ps->nufft, st);

	if (ps->conf.precond) {	// z0 = M(b); the first direction is p = z0

		int nd = 0;
		const char* e = getenv("BNUFFT_FCG_FUSE");
		ps->fcg_fused = (1 == ps->conf.precond) && (1 == ps->fcg_m) && ps->fcg_fold
				&& (0 != precond_cluster_size(ps->nufft->op.g)) && !(e && (0 == strcmp(e, "0")));

		if (ps->fcg_fused) {	// p0 = z0 and its partials, from the cluster preconditioner

			PcDir d = { ps->scal, 0, 1, ps->rs_part, ps->nparts, ps->pbuf[1], ps->r, ps->pr_part, ps->pp_part };
			TRY(pics_precond_circ(ps, ps->r, ps->z, nullptr, nullptr, &nd, st, &d));
			ps->ndir = nd;

		} else {

			TRY(pics_precond(ps, ps->r, ps->z, nullptr, nullptr, &nd, st));
		}

		if (nd > ps->max_row_blocks)
			return fail(BNUFFT_ERR_ARG, "internal: partial arrays too small");

		ps->ndots = nd;		// the folded iteration's <z, A p> partials per launch
	}

	if (ps->conf.maxiter > 0) {

		if (graph) {

			if (!ps->cg_exec)
				TRY(capture_cg_loop(ps));

			CUDA_TRY(cudaGraphLaunch(ps->cg_exec, st));
			ps->last_graph = true;

		} else {

			for (int it = 0; it < ps->conf.maxiter; it++)
				TRY(pics_any_iteration(ps, it, st));
		}
	}

	k_cg_finish<<<1, RED_THREADS, 0, st>>>(ps->scal, ps->conf.maxiter, ps->rs_part, ps->nparts);
	LAUNCHED();

	if (ps->conf.rescale) {

		k_scale_dev<<<nb, RED_THREADS, 0, st>>>(out, ps->x, ps->npix, &ps->scal->scale);
		LAUNCHED();

	} else {

		CUDA_TRY(cudaMemcpyAsync(out, ps->x, ib, cudaMemcpyDeviceToDevice, st));
	}

	return BNUFFT_OK;
}

extern "C" int bnufft_pics_run(bnufft_pics_t ps, void* img, const void* ksp, void* stream)
{
	cudaStream_t st = S(stream);
	size_t kb = sizeof(float2) * ps->M * ps->C;
	size_t ib = sizeof(float2) * ps->npix;
	Staged ki, io;
	TRY(stage_in(ki, ksp, kb, st));
	TRY(stage_out_alloc(io, img, ib, st));
	long launches0 = g_launches.load();
	TRY(pics_solve(ps, (const float2*)ki.dev, (float2*)io.dev, st, cg_graph_enabled()));
	ps->last_host_kernels = g_launches.load() - launches0;

	if (!ps->run_done)
		CUDA_TRY(cudaEventCreateWithFlags(&ps->run_done, cudaEventDisableTiming));

	CUDA_TRY(cudaEventRecord(ps->run_done, st));
	return stage_out_copy(io, img, ib, st);
}

// ----------------------------------------------------------------------------
// batches of independent reconstructions as one graph
// ----------------------------------------------------------------------------

struct bnufft_batch_s {

	std::vector<bnufft_pics_t> models;
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	long kernels = 0;		// kernel nodes in the graph
};

extern "C" void bnufft_batch_free(bnufft_batch_t b)
{
	if (!b)
		return;

	if (b->exec)
		cudaGraphExecDestroy(b->exec);

	if (b->graph)
		cudaGraphDestroy(b->graph);

	delete b;
}

extern "C" int bnufft_batch_create(bnufft_batch_t* out, const bnufft_pics_t* models, int n, void* const* imgs,
		const void* const* ksps, void* stream)
{
	cudaStream_t st = S(stream);

	if (!out || !models || !imgs || !ksps || (n < 1))
		return fail(BNUFFT_ERR_ARG, "null argument or empty batch");

	for (int p = 0; p < n; p++) {

		if (!models[p])
			return fail(BNUFFT_ERR_ARG, "batch model %d is null", p);

		if (!on_device(imgs[p]) || !on_device(ksps[p]))
			return fail(BNUFFT_ERR_ARG, "batch problem %d: images and k-space must be device memory", p);

		if (models[p]->conf.tol > 0.f)
			return fail(BNUFFT_ERR_UNSUPPORTED, "batch problem %d: batches run a fixed iteration count (tol 0)", p);

		OpCtx& op = models[p]->nufft->op;
		TRY(alloc_work(op.w, op.g, models[p]->C, st));

		if (models[p]->nufft->embed)
			TRY(alloc_work(models[p]->nufft->toe.w, models[p]->nufft->toe.g, models[p]->C, st));

		// the captured solves do not wait for the PSF's stream: it is done first
		if (models[p]->nufft->psf_ev)
			CUDA_TRY(cudaEventSynchronize(models[p]->nufft->psf_ev));
	}

	CUDA_TRY(cudaStreamSynchronize(st));

	auto b = new bnufft_batch_s();
	b->models.assign(models, models + n);
	cudaStream_t cap = nullptr;
	int s = BNUFFT_OK;
	cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);

	if (cudaSuccess == e)
		e = cudaGraphCreate(&b->graph, 0);

	if (cudaSuccess != e)
		s = fail(BNUFFT_ERR_CUDA, "batch graph: %s", cudaGetErrorString(e));

	// every problem's solve is captured into its own graph and added as a
	// child node without dependencies: the problems run concurrently
	for (int p = 0; (p < n) && (BNUFFT_OK == s); p++) {

		cudaGraph_t gp = nullptr;
		e = cudaGraphCreate(&gp, 0);

		if (cudaSuccess == e)
			e = cudaStreamBeginCaptureToGraph(cap, gp, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);

		if (cudaSuccess != e) {

			s = fail(BNUFFT_ERR_CUDA, "batch capture %d: %s", p, cudaGetErrorString(e));

			if (gp)
				cudaGraphDestroy(gp);

			break;
		}

		long before = g_launches.load();
		s = pics_solve(models[p], (const float2*)ksps[p], (float2*)imgs[p], cap, false);
		long k = g_launches.load() - before;
		g_launches.fetch_sub(k);	// captured, not launched
		b->kernels += k;
		cudaGraph_t got = nullptr;
		e = cudaStreamEndCapture(cap, &got);

		if ((BNUFFT_OK == s) && (cudaSuccess != e))
			s = fail(BNUFFT_ERR_CUDA, "batch capture %d: %s", p, cudaGetErrorString(e));

		if (BNUFFT_OK == s) {

			cudaGraphNode_t node;
			e = cudaGraphAddChildGraphNode(&node, b->graph, nullptr, 0, gp);

			if (cudaSuccess != e)
				s = fail(BNUFFT_ERR_CUDA, "batch graph node %d: %s", p, cudaGetErrorString(e));
		}

		cudaGraphDestroy(gp);	// the child node holds its own copy
	}

	if (BNUFFT_OK == s) {

		e = cudaGraphInstantiate(&b->exec, b->graph, 0);

		if (cudaSuccess != e)
			s = fail(BNUFFT_ERR_CUDA, "batch instantiate: %s", cudaGetErrorString(e));
	}

	if (cap)
		cudaStreamDestroy(cap);

	if (BNUFFT_OK != s) {

		std::string msg = g_err;
		bnufft_batch_free(b);
		g_err = msg;
		return s;
	}

	*out = b;
	return BNUFFT_OK;
}

extern "C" int bnufft_batch_run(bnufft_batch_t b, void* stream)
{
	CUDA_TRY(cudaGraphLaunch(b->exec, S(stream)));
	g_launches.fetch_add(b->kernels, std::memory_order_relaxed);
	return BNUFFT_OK;
}

extern "C" long bnufft_batch_kernels(bnufft_batch_t b) { return b ? b->kernels : 0; }

extern "C" int bnufft_pics_set_precnet(bnufft_pics_t ps, bnufft_precnet_t net, void* stream)
{
	cudaStream_t st = S(stream);

	if (!ps || (2 != ps->conf.precond))
		return fail(BNUFFT_ERR_ARG, "the model was not created with precond 2");

	if (ps->nufft->op.g.N[2] > 1)
		return fail(BNUFFT_ERR_UNSUPPORTED, "the learned preconditioner is 2D");

	ps->net = net;

	for (auto& a : ps->nact)
		if (!a)
			CUDA_TRY(cudaMallocAsync(&a, sizeof(bf16) * NET_C * ps->npix, st));

	if (!ps->mcn_part)
		CUDA_TRY(cudaMallocAsync(&ps->mcn_part, sizeof(double) * ps->max_row_blocks, st));

	return BNUFFT_OK;
}

extern "C" int bnufft_pics_set_iter(bnufft_pics_t ps, int maxiter, float tol)
{
	if (!ps || (maxiter < 0) || !(tol >= 0.f))
		return fail(BNUFFT_ERR_ARG, "bad iteration limit or tolerance");

	ps->conf.maxiter = maxiter;
	ps->conf.tol = tol;
	return BNUFFT_OK;
}

// b = A^H y / scale (the right-hand side the solve uses)
extern "C" int bnufft_pics_rhs(bnufft_pics_t ps, void* b, const void* ksp, void* stream)
{
	cudaStream_t st = S(stream);
	size_t kb = sizeof(float2) * ps->M * ps->C;
	size_t ib = sizeof(float2) * ps->npix;
	Staged ki, bo;
	TRY(stage_in(ki, ksp, kb, st));
	TRY(stage_out_alloc(bo, b, ib, st));
	TRY(pics_prologue(ps, (const float2*)ki.dev, st));
	CUDA_TRY(cudaMemcpyAsync(bo.dev, ps->b, ib, cudaMemcpyDeviceToDevice, st));
	return stage_out_copy(bo, b, ib, st);
}

// z = M(r) with the model's preconditioner (precond 1 or 2)
extern "C" int bnufft_pics_precond(bnufft_pics_t ps, void* z, const void* r, void* stream)
{
	cudaStream_t st = S(stream);

	if (!ps->conf.precond)
		return fail(BNUFFT_ERR_ARG, "the model has no preconditioner");

	size_t ib = sizeof(float2) * ps->npix;
	Staged ri, zo;
	TRY(stage_in(ri, r, ib, st));
	TRY(stage_out_alloc(zo, z, ib, st));
	OpCtx& op = ps->nufft->op;
	TRY(alloc_work(op.w, op.g, ps->C, st));
	k_norm_scalars<<<1, RED_THREADS, 0, st>>>((const float2*)ri.dev, ps->npix, ps->scal);
	LAUNCHED();
	TRY(pics_precond(ps, (const float2*)ri.dev, (float2*)zo.dev, nullptr, nullptr, nullptr, st));
	return stage_out_copy(zo, z, ib, st);
}

extern "C" int bnufft_pics_kernels(bnufft_pics_t ps, long* kernels, void* stream)
{
	CgScalars h;
	CUDA_TRY(cudaMemcpyAsync(&h, ps->scal, sizeof h, cudaMemcpyDeviceToHost, S(stream)));
	CUDA_TRY(cudaStreamSynchronize(S(stream)));
	*kernels = ps->last_host_kernels + (ps->last_graph ? (long)h.it * ps->body_kernels : 0L);
	return BNUFFT_OK;
}

extern "C" int bnufft_pics_stats(bnufft_pics_t ps, int* iters, double* rel_resid, float* scaling, void* stream)
{
	CgScalars h;
	CUDA_TRY(cudaMemcpyAsync(&h, ps->scal, sizeof h, cudaMemcpyDeviceToHost, S(stream)));
	CUDA_TRY(cudaStreamSynchronize(S(stream)));

	if (iters)
		*iters = h.iters;

	if (rel_resid)
		*rel_resid = (h.b2 > 0.) ? sqrt(h.rs[h.iters & 1] / h.b2) : 0.;	// rs of the last completed iteration

	if (scaling)
		*scaling = h.scale;

	return BNUFFT_OK;
}

extern "C" void bnufft_pics_free(bnufft_pics_t ps)
{
	if (!ps)
		return;

	cudaStream_t st = ps->nufft ? ps->nufft->st0 : nullptr;
	reap_graves();

	// the stream-ordered frees below follow the last run, on whatever stream
	// it was, and the auxiliary stream's set-up work (the preconditioner
	// spectrum is written there)
	if (ps->run_done)
		cudaStreamWaitEvent(st, ps->run_done, 0);

	if (ps->nufft)
		psf_wait(ps->nufft, st);

	if (ps->cg_exec && ps->run_done) {

		LoopGraph lg = { ps->cg_dev, ps->cg_graph, ps->cg_body, ps->cg_loop, ps->cg_exec, ps->run_done };
		bool kept = false;
		ps->run_done = nullptr;

		{
			std::lock_guard<std::mutex> lock(g_loop_mutex);

			if (g_loop_pool.size() < LOOP_POOL_MAX) {

				g_loop_pool.push_back(lg);
				kept = true;
			}
		}

		if (!kept)
			bury(lg);

	} else {

		if (ps->cg_exec)
			cudaGraphExecDestroy(ps->cg_exec);

		if (ps->cg_graph)
			cudaGraphDestroy(ps->cg_graph);
	}

	if (ps->run_done)
		cudaEventDestroy(ps->run_done);

	void* bufs[] = { ps->sens, ps->part, ps->x, ps->r, ps->pbuf[0], ps->pbuf[1], ps->b, ps->kbuf, ps->mag, ps->sel,
			 ps->pap_part, ps->pp_part, ps->rs_part, ps->scal, ps->z, ps->p_ring, ps->ap_ring,
			 ps->dots_part, ps->pr_part, ps->nact[0], ps->nact[1], ps->mcn_part, ps->pinv_pad };

	for (void* b : bufs)
		if (b)
			cudaFreeAsync(b, st);

	bnufft_free(ps->nufft);
	delete ps;
}

extern "C" const char* bnufft_last_error(void) { return g_err.c_str(); }

extern "C" int bnufft_prof_start(const char* kind)
{
	std::lock_guard<std::mutex> lock(g_prof_mutex);

	for (auto& e : g_prof_events) {

		cudaEventDestroy(e.first);
		cudaEventDestroy(e.second);
	}

	g_prof_events.clear();
	g_prof_target = kind ? kind : "";
	g_prof_active.store(!g_prof_target.empty());
	return BNUFFT_OK;
}

extern "C" int bnufft_prof_stop(double* total_ms, long* launches)
{
	std::lock_guard<std::mutex> lock(g_prof_mutex);
	double tot = 0.;

	for (auto& e : g_prof_events) {

		float ms = 0.f;
		CUDA_TRY(cudaEventSynchronize(e.second));
		CUDA_TRY(cudaEventElapsedTime(&ms, e.first, e.second));
		tot += ms;
	}

	if (total_ms)
		*total_ms = tot;

	if (launches)
		*launches = (long)g_prof_events.size();

	for (auto& e : g_prof_events) {

		cudaEventDestroy(e.first);
		cudaEventDestroy(e.second);
	}

	g_prof_events.clear();
	g_prof_target.clear();
	g_prof_active.store(false);
	return BNUFFT_OK;
}

extern "C" long bnufft_launch_count(void) { return g_launches.load(); }

// ----------------------------------------------------------------------------
// Allocation-free 2D forward NUFFT (C ABI: bnufft_forward2d_noalloc)
// ----------------------------------------------------------------------------
//
// For callers that cannot allocate device memory while they run: a scanner's
// real-time reconstruction process that reserves its whole device budget up
// front, or code that must not pay cudaMalloc's implicit device-wide
// synchronisation (or risk its failure under memory pressure) in the middle
// of a stream of work. Everything this entry point needs beyond the caller's
// trajectory, image and k-space buffers lives in one file-scope device array,
// g_noalloc_scratch, which every GPU that loads the library holds until the
// process exits (NA_BYTES, about 7.4 MB).
//
// Limits: 2D images X x Y with X, Y in {8, 16, ..., 256}, at most NA_MAX_M
// samples, one coil. Larger requests return BNUFFT_ERR_ARG.
//
// The first call on a device does the set-up: it takes the array's device
// address with cudaGetSymbolAddress (the array's name in host code is only a
// host-side stand-in), copies in the Kaiser-Bessel, twiddle and roll-off
// tables, built on the host by the same functions as a plan's (kb_precompute,
// twiddles_host, rolloff_host), and synchronises the caller's stream once.
// Make that first call before any stream capture. A cudaDeviceReset between
// calls is not supported: it would drop the tables without this library
// noticing.
//
// All calls share the one array and every call overwrites the regions it
// uses (trajectory copy, row-transformed buffer, grid); the tables are only
// read. So nothing needs clearing between calls; calls whose work overlaps
// on the GPU (different streams, or another thread) race on the array and
// must be serialised by the caller.

enum : long {

	NA_MIN_N = 8,
	NA_MAX_N = 256,
	NA_NSIDES = 6,							// 8, 16, ..., 256
	NA_ROLL_N = 512,						// floats per roll-off table set
	NA_MAX_M = 262144,
	NA_TRAJ_OFF = 0,						// float4[NA_MAX_M]
	NA_T1_OFF = NA_TRAJ_OFF + 16L * NA_MAX_M,			// float2[2N x N]
	NA_GRID_OFF = NA_T1_OFF + 8L * (2 * NA_MAX_N) * NA_MAX_N,	// float2[2N x 2N]
	NA_TW_OFF = NA_GRID_OFF + 8L * (2 * NA_MAX_N) * (2 * NA_MAX_N),	// float2[1024]: L = 16..512 back to back
	NA_KB_OFF = NA_TW_OFF + 8L * 1024,				// float[1024]
	NA_AX_OFF = NA_KB_OFF + 4L * 1024,				// float[NA_ROLL_N]: ax of X = 8..256 back to back
	NA_AYZ_OFF = NA_AX_OFF + 4L * NA_ROLL_N,			// float[NA_NSIDES][NA_ROLL_N]: ayz of (X, Y)
	NA_BYTES = NA_AYZ_OFF + 4L * NA_NSIDES * NA_ROLL_N,
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

static std::mutex g_na_mutex;
static unsigned char* g_na_base[64];

// twiddle table of length L (power of two, 16..512) inside the scratch table block
static long na_tw_offset(int L) { return L - 16; }

// roll-off tables of an image side n (power of two, 8..256): ax at
// na_roll_offset(X), ayz of (X, Y) in the table set of X at na_roll_offset(Y)
static long na_roll_offset(long n) { return n - NA_MIN_N; }

static int na_log2(long n)
{
	int k = 0;

	while ((1L << k) < n)
		k++;

	return k;
}

template <int L>
static int na_rows(const float2* img, const float* ax, const float* ayz, int X, int Y, float2* out,
		const float2* tw, cudaStream_t st)
{
	constexpr int B = 16;
	size_t smem = rows_smem(L, B);
	TRY(prep_kernel(k_rows_fwd<L, B, false>, smem));
	k_rows_fwd<L, B, false><<<(unsigned)((Y + B - 1) / B), B * L / 8, smem, st>>>(img, nullptr, ax, ayz, X, Y, Y, out, tw, nullptr, Dft{L, nullptr, nullptr, nullptr});
	LAUNCHED();
	return BNUFFT_OK;
}

template <int L>
static int na_cols(const float2* t1, int G0, int Y, float2* grid, const float2* tw, cudaStream_t st)
{
	constexpr int B = 16;
	size_t smem = pass_smem(L, B);
	TRY(prep_kernel(k_cols<L, B, 0, false>, smem));
	dim3 grid_dim((unsigned)((G0 + B - 1) / B), 1);
	k_cols<L, B, 0, false><<<grid_dim, B * L / 8, smem, st>>>(t1, G0, (long)G0 * Y, Y, 1, grid, G0, (long)G0 * L, L, 0,
			G0, nullptr, 0, 1, 0, tw, nullptr, Dft{L, nullptr, nullptr, nullptr});
	LAUNCHED();
	return BNUFFT_OK;
}

#define NA_DISPATCH(L, CALL) \
	switch (L) { \
	case 16: { constexpr int LL = 16; return CALL; } \
	case 32: { constexpr int LL = 32; return CALL; } \
	case 64: { constexpr int LL = 64; return CALL; } \
	case 128: { constexpr int LL = 128; return CALL; } \
	case 256: { constexpr int LL = 256; return CALL; } \
	case 512: { constexpr int LL = 512; return CALL; } \
	default: return fail(BNUFFT_ERR_ARG, "allocation-free NUFFT: grid length %d", L); }

static int na_setup(unsigned char** base, cudaStream_t st)
{
	int dev;
	CUDA_TRY(cudaGetDevice(&dev));

	if ((dev < 0) || (dev >= 64))
		return fail(BNUFFT_ERR_ARG, "device index %d", dev);

	std::lock_guard<std::mutex> lock(g_na_mutex);

	if (g_na_base[dev]) {

		*base = g_na_base[dev];
		return BNUFFT_OK;
	}

	void* p = nullptr;
	cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);

	if ((cudaSuccess != e) || (nullptr == p))
		return fail(BNUFFT_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));

	// the tables a plan would build, on the host, into one host block that
	// mirrors the scratch's table region [NA_TW_OFF, NA_BYTES)
	std::vector<unsigned char> h(NA_BYTES - NA_TW_OFF, 0);
	auto at = [&](long off) { return h.data() + (off - NA_TW_OFF); };	// scratch offset -> host block

	for (int L = 16; L <= 512; L *= 2)
		twiddles_host(L, (float2*)at(NA_TW_OFF) + na_tw_offset(L));

	kb_precompute(kernel_beta(2.f, 6.f), KB_TABLE_N, (float*)at(NA_KB_OFF));

	for (long X = NA_MIN_N; X <= NA_MAX_N; X *= 2)
		for (long Y = NA_MIN_N; Y <= NA_MAX_N; Y *= 2) {

			const int n[3] = { (int)X, (int)Y, 1 };
			float* ayz = (float*)at(NA_AYZ_OFF) + NA_ROLL_N * (na_log2(X) - na_log2(NA_MIN_N)) + na_roll_offset(Y);
			std::vector<float> ax(X);
			rolloff_host(n, 2.f, 6.f, ax.data(), ayz);
			std::memcpy((float*)at(NA_AX_OFF) + na_roll_offset(X), ax.data(), sizeof(float) * X);
		}

	unsigned char* b = (unsigned char*)p;
	CUDA_TRY(cudaMemcpyAsync(b + NA_TW_OFF, h.data(), h.size(), cudaMemcpyHostToDevice, st));
	CUDA_TRY(cudaStreamSynchronize(st));	// tables ready before any other stream uses them (and h is freed)
	g_na_base[dev] = b;
	*base = b;
	return BNUFFT_OK;
}

extern "C" int bnufft_forward2d_noalloc(long X, long Y, long M, const void* traj, const void* img, void* ksp, void* stream)
{
	cudaStream_t st = S(stream);

	for (long n : { X, Y })
		if ((n < NA_MIN_N) || (n > NA_MAX_N) || (0 != (n & (n - 1))))
			return fail(BNUFFT_ERR_ARG, "allocation-free NUFFT: image side %ld (powers of two %ld..%ld)", n,
					(long)NA_MIN_N, (long)NA_MAX_N);

	if ((M < 1) || (M > NA_MAX_M))
		return fail(BNUFFT_ERR_ARG, "allocation-free NUFFT: %ld samples (at most %ld)", M, (long)NA_MAX_M);

	if (!traj || !img || !ksp || !on_device(traj) || !on_device(img) || !on_device(ksp))
		return fail(BNUFFT_ERR_ARG, "allocation-free NUFFT: traj, img and ksp must be device pointers");

	unsigned char* base = nullptr;
	TRY(na_setup(&base, st));

	float4* ntraj = (float4*)(base + NA_TRAJ_OFF);
	float2* t1 = (float2*)(base + NA_T1_OFF);
	float2* grid = (float2*)(base + NA_GRID_OFF);
	const float2* tw = (const float2*)(base + NA_TW_OFF);
	const float* kb = (const float*)(base + NA_KB_OFF);
	const float* ax = (const float*)(base + NA_AX_OFF) + na_roll_offset(X);
	const float* ayz = (const float*)(base + NA_AYZ_OFF) + NA_ROLL_N * (na_log2(X) - na_log2(NA_MIN_N)) + na_roll_offset(Y);

	const int G0 = (int)(2 * X), G1 = (int)(2 * Y);

	k_traj_convert<<<vec_blocks(M), RED_THREADS, 0, st>>>(ntraj, (const float2*)traj, M, 1.f);
	LAUNCHED();

	auto rowsf = [&]() -> int { NA_DISPATCH(G0, (na_rows<LL>((const float2*)img, ax, ayz, (int)X, (int)Y, t1, tw + na_tw_offset(LL), st))); };
	TRY(rowsf());

	auto colsf = [&]() -> int { NA_DISPATCH(G1, (na_cols<LL>(t1, G0, (int)Y, grid, tw + na_tw_offset(LL), st))); };
	TRY(colsf());

	GridGeom gg;
	gg.N[0] = (int)X;
	gg.N[1] = (int)Y;
	gg.N[2] = 1;
	gg.G[0] = G0;
	gg.G[1] = G1;
	gg.G[2] = 1;
	gg.gsz = (long)G0 * G1;
	gg.hw = 3.f;
	gg.periodic = 0;
	k_degrid<<<(unsigned)((M + 127) / 128), 128, 0, st>>>(ntraj, M, gg, 1, 1, grid, (float2*)ksp, kb);
	LAUNCHED();
	return BNUFFT_OK;
}

// CG for an operator applied by the caller (bnufft_cg_*)
#include "cgext.cuh"

// ESPIRiT calibration (include/bespirit.h)
#include "espirit.cuh"
