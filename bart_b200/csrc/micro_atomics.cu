// Atomic-add throughput on this GPU: the roofline of a scatter that adds
// with atomics (the NUFFT adjoint's gridding). Every thread adds 1 to random
// addresses inside a span of 512 or 4096 elements, in shared memory (float,
// int32, uint64) or in global memory (float, float2, float4 vector atomics;
// the span repeated per group of blocks, L2-resident). Prints one line per
// case: time and atomic operations per second.
#include <cstdio>
#include <cuda_runtime.h>

__device__ __forceinline__ unsigned mix(unsigned x)
{
	x ^= x >> 16;
	x *= 0x7feb352dU;
	x ^= x >> 15;
	x *= 0x846ca68bU;
	x ^= x >> 16;
	return x;
}

enum { SPAN_MAX = 4096, GROUPS = 64 };

template <int KIND>
__global__ void k_atomics(float* __restrict__ gout, int iters, int span, float4* __restrict__ g4)
{
	__shared__ float sf[SPAN_MAX];
	__shared__ int si[SPAN_MAX];
	__shared__ unsigned long long su[SPAN_MAX / 2];

	for (int i = threadIdx.x; i < SPAN_MAX; i += blockDim.x) {

		sf[i] = 0.f;
		si[i] = 0;
		su[i / 2] = 0ULL;
	}

	__syncthreads();
	unsigned s = mix(blockIdx.x * 1024u + threadIdx.x);

	for (int it = 0; it < iters; it++) {

		s = mix(s + (unsigned)it);
		int a = (int)(s % (unsigned)span);	// span <= SPAN_MAX

		if (0 == KIND) atomicAdd(&sf[a], 1.f);
		if (1 == KIND) atomicAdd(&si[a], 1);
		if (2 == KIND) atomicAdd(&su[a / 2], 1ULL);
		if (3 == KIND) atomicAdd(&gout[(blockIdx.x % GROUPS) * SPAN_MAX + a], 1.f);
		if (4 == KIND) atomicAdd((float2*)&g4[(blockIdx.x % GROUPS) * SPAN_MAX + a], make_float2(1.f, 1.f));
		if (5 == KIND) atomicAdd(&g4[(blockIdx.x % GROUPS) * SPAN_MAX + a], make_float4(1.f, 1.f, 1.f, 1.f));
	}

	__syncthreads();
	float acc = 0.f;

	for (int i = threadIdx.x; i < SPAN_MAX; i += blockDim.x)
		acc += sf[i] + (float)si[i] + (float)su[i / 2];

	if (-1.f == acc)	// keeps the shared-memory results live
		gout[0] = acc;
}

int main()
{
	float* g = nullptr;
	float4* g4 = nullptr;

	if ((cudaSuccess != cudaMalloc(&g, sizeof(float) * GROUPS * SPAN_MAX)) ||
			(cudaSuccess != cudaMalloc(&g4, sizeof(float4) * GROUPS * SPAN_MAX)))
		return 1;

	cudaMemset(g, 0, sizeof(float) * GROUPS * SPAN_MAX);
	cudaMemset(g4, 0, sizeof(float4) * GROUPS * SPAN_MAX);
	const int iters = 4096, blocks = 148 * 4, threads = 256;
	const char* names[] = { "shared f32", "shared i32", "shared u64", "global f32", "global float2", "global float4" };
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);

	for (int span : { 4096, 512 }) {

		for (int kind = 0; kind < 6; kind++) {

			float ms = 0.f;

			for (int rep = 0; rep < 2; rep++) {

				cudaEventRecord(e0);

				switch (kind) {
				case 0: k_atomics<0><<<blocks, threads>>>(g, iters, span, g4); break;
				case 1: k_atomics<1><<<blocks, threads>>>(g, iters, span, g4); break;
				case 2: k_atomics<2><<<blocks, threads>>>(g, iters, span, g4); break;
				case 3: k_atomics<3><<<blocks, threads>>>(g, iters, span, g4); break;
				case 4: k_atomics<4><<<blocks, threads>>>(g, iters, span, g4); break;
				default: k_atomics<5><<<blocks, threads>>>(g, iters, span, g4); break;
				}

				cudaEventRecord(e1);
				cudaEventSynchronize(e1);
				cudaEventElapsedTime(&ms, e0, e1);
			}

			double n = (double)iters * blocks * threads;
			printf("{\"span\": %d, \"kind\": \"%s\", \"ms\": %.4f, \"g_atomics_per_s\": %.1f, \"status\": \"%s\"}\n",
				span, names[kind], ms, n / ms / 1e6, cudaGetErrorString(cudaGetLastError()));
		}
	}

	cudaFree(g);
	cudaFree(g4);
	return 0;
}
