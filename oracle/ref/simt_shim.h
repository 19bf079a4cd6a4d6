/*
 * simt_shim.h -- lets the reference's CUDA kernel source (cuda/*.cu of
 * AutoDock-GPU) compile and run as host C++ so that it can serve as the
 * parity oracle.  TEST INFRASTRUCTURE ONLY: nothing in the product links it.
 *
 * Execution model (faithful to CUDA for the constructs the reference uses):
 *   - a "block" of blockDim.x threads is run as blockDim.x cooperative fibers
 *     (ucontext) on one OS thread;
 *   - __syncthreads() parks a fiber until every live fiber of the block has
 *     arrived;
 *   - __shfl_sync / __any_sync park a fiber until every live lane of its
 *     warp (32 lanes) has deposited its value, so warp collectives see the
 *     same values and the same butterfly order as on the GPU;
 *   - __shared__ variables are function-local `static thread_local`, i.e.
 *     shared by the fibers of one block and private to each OS thread (blocks
 *     of one launch may run on several OS threads, see adgpu_ref_launch);
 *   - atomics are plain read-modify-writes: fibers only switch at the
 *     collectives above, so every atomic is indivisible.
 * Because each emulated thread keeps its own threadIdx, the per-thread LCG
 * states (prng_states[blockIdx.x*blockDim.x+threadIdx.x], cuda/auxiliary_genetic.cu:37)
 * are consumed exactly as on the device.
 *
 * The only deliberate deviation: transcendental/fast-math intrinsics map to
 * the precise libm functions (__powf -> powf, sin -> sinf, ...).
 */
#ifndef ADGPU_SIMT_SHIM_H
#define ADGPU_SIMT_SHIM_H

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <cfloat>
#include <functional>
#include <sys/types.h>

using std::sqrt; using std::sin; using std::cos; using std::floor; using std::fabs;
using std::copysign; using std::atan2; using std::pow; using std::acos;

/* ---- CUDA qualifiers --------------------------------------------------- */
#define __device__
#define __global__
#define __host__
#define __forceinline__ inline
#define __constant__
#define __shared__ static thread_local
#define __launch_bounds__(...)
#define __restrict__
/* kernels.cu carries two unused PTX helpers; neutralise their inline asm */
#define asm(...) (void)0

/* ---- vector types ------------------------------------------------------ */
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
struct int3   { int x, y, z; };
struct uint3_ { unsigned int x, y, z; };
static inline float3 make_float3(float x, float y, float z) { float3 r = {x, y, z}; return r; }
static inline float4 make_float4(float x, float y, float z, float w) { float4 r = {x, y, z, w}; return r; }

/* ---- thread coordinates (set by the fiber scheduler) -------------------- */
extern thread_local uint3_ adgpu_sim_threadIdx;
extern thread_local uint3_ adgpu_sim_blockIdx;
extern thread_local uint3_ adgpu_sim_blockDim;
#define threadIdx adgpu_sim_threadIdx
#define blockIdx  adgpu_sim_blockIdx
#define blockDim  adgpu_sim_blockDim

/* ---- collectives --------------------------------------------------------- */
void adgpu_sim_syncthreads();
uint32_t adgpu_sim_shfl_bits(uint32_t bits, int src_lane);
int adgpu_sim_any(int pred);
#define __syncthreads() adgpu_sim_syncthreads()
#define __threadfence() ((void)0)
static inline float __shfl_sync(unsigned, float v, int src) {
	uint32_t b; memcpy(&b, &v, 4); b = adgpu_sim_shfl_bits(b, src); float r; memcpy(&r, &b, 4); return r;
}
static inline int __shfl_sync(unsigned, int v, int src) {
	return (int)adgpu_sim_shfl_bits((uint32_t)v, src);
}
static inline unsigned __shfl_sync(unsigned, unsigned v, int src) {
	return adgpu_sim_shfl_bits(v, src);
}
static inline int __any_sync(unsigned, int pred) { return adgpu_sim_any(pred); }
static inline int __any_sync(unsigned, bool pred) { return adgpu_sim_any(pred ? 1 : 0); }

static inline int atomicAdd(int* p, int v) { int o = *p; *p = o + v; return o; }
static inline unsigned atomicAdd(unsigned* p, unsigned v) { unsigned o = *p; *p = o + v; return o; }
static inline float atomicAdd(float* p, float v) { float o = *p; *p = o + v; return o; }
static inline float atomicAdd(volatile float* p, float v) { float o = *p; *p = o + v; return o; }

/* ---- math intrinsics (precise host equivalents) ------------------------- */
#define __powf(a, b) powf((float)(a), (float)(b))
#define __fdividef(a, b) ((a) / (b))
static inline float norm3df(float a, float b, float c) { return sqrtf(a * a + b * b + c * c); }
static inline float rnorm3df(float a, float b, float c) { return 1.0f / sqrtf(a * a + b * b + c * c); }

/* ---- CUDA runtime surface used by the reference's kernel API TU --------- */
typedef int cudaError_t;
#define cudaSuccess 0
static inline const char* cudaGetErrorString(cudaError_t) { return "emulated"; }
static inline cudaError_t cudaDeviceReset() { return 0; }
static inline cudaError_t cudaDeviceSynchronize() { return 0; }
static inline cudaError_t cudaGetLastError() { return 0; }
template <class T> static inline cudaError_t cudaMemcpyToSymbol(T& sym, const void* src, size_t n) {
	memcpy((void*)&sym, src, n); return 0;
}
template <class T> static inline cudaError_t cudaMemcpyFromSymbol(void* dst, const T& sym, size_t n) {
	memcpy(dst, (const void*)&sym, n); return 0;
}

/* ---- launch --------------------------------------------------------------
 * Runs `blocks` blocks of `threads` emulated threads, each calling `body`.
 * Blocks are distributed over ADGPU_REF_THREADS OS threads (default 1);
 * the reference's kernels touch disjoint global memory per block, except
 * for per-run counters that are only written by kernel2 (one block per run).
 */
void adgpu_ref_launch(unsigned blocks, unsigned threads, const std::function<void()>& body);

#endif
