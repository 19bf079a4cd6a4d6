// fp32_peak.cu -- bench-only library (libadgpu_probe.so, not part of
// libadgpu_b200): the measured FP32 FMA throughput of the current device,
// independent FMA chains on every SM, the denominator bench.py uses for the
// scorer's roofline fraction (the driver's peak file carries HBM and bf16
// tensor figures only).
//
//   int adgpu_probe_fp32_peak(float* device_scratch, size_t n_floats, float* tflops)
//   device_scratch: 2048 floats per SM; returns 0, 1 (bad argument) or the
//   CUDA error code.
#include <cuda_runtime.h>
#include <cstddef>

__global__ void __launch_bounds__(256) fma_probe_kernel(float* out, int iters, float m, float c)
{
	float a0 = threadIdx.x * 1e-7f, a1 = a0 + 1e-7f, a2 = a0 + 2e-7f, a3 = a0 + 3e-7f;
	float a4 = a0 + 4e-7f, a5 = a0 + 5e-7f, a6 = a0 + 6e-7f, a7 = a0 + 7e-7f;
	for (int i = 0; i < iters; i++) {
#pragma unroll
		for (int k = 0; k < 8; k++) {
			a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
			a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
		}
	}
	out[blockIdx.x * blockDim.x + threadIdx.x] = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
}

extern "C" int adgpu_probe_fp32_peak(float* device_scratch, size_t n_floats, float* tflops)
{
	if (!device_scratch || !tflops) return 1;
	int dev = 0, sms = 0;
	cudaError_t e = cudaGetDevice(&dev);
	if (e != cudaSuccess) return (int)e;
	e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	if (e != cudaSuccess) return (int)e;
	const int threads = 256, blocks = sms * 8;
	if (n_floats < (size_t)threads * blocks) return 1;
	const int iters = 4096;
	cudaEvent_t a, b;
	if ((e = cudaEventCreate(&a)) != cudaSuccess) return (int)e;
	if ((e = cudaEventCreate(&b)) != cudaSuccess) { cudaEventDestroy(a); return (int)e; }
	fma_probe_kernel<<<blocks, threads>>>(device_scratch, 64, 1.0000001f, 1e-7f);   // warm-up
	float best = 1e30f;
	for (int rep = 0; rep < 5; rep++) {
		cudaEventRecord(a);
		fma_probe_kernel<<<blocks, threads>>>(device_scratch, iters, 1.0000001f, 1e-7f);
		cudaEventRecord(b);
		cudaEventSynchronize(b);
		float ms = 0;
		cudaEventElapsedTime(&ms, a, b);
		if (ms < best) best = ms;
	}
	cudaEventDestroy(a);
	cudaEventDestroy(b);
	e = cudaGetLastError();
	if (e != cudaSuccess) return (int)e;
	const double flops = 2.0 * 8.0 * 8.0 * iters * (double)threads * blocks;
	*tflops = (float)(flops / (best * 1e-3) / 1e12);
	return 0;
}
