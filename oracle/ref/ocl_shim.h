/*
 * ocl_shim.h -- lets the reference's OpenCL device source (device/*.cl of
 * AutoDock-GPU: the FIRE local search, kernel_fire.cl, and the functions it
 * calls) compile and run as host C++ on the same cooperative-fiber SIMT
 * emulator as its CUDA kernels (simt_shim.cpp).  TEST INFRASTRUCTURE ONLY:
 * nothing in the product links it.
 *
 * Model:
 *   - a work-group of get_local_size(0) work-items runs as that many fibers on
 *     one OS thread; barrier() parks a fiber until every live fiber of the
 *     group has arrived (the emulator's block barrier);
 *   - __local variables declared in a kernel body become function-level
 *     `static thread_local` (the recipe in oracle/Makefile rewrites those
 *     declarations after preprocessing; __local on pointers is dropped), i.e.
 *     shared by the fibers of one group and private to each OS thread;
 *   - atomics are plain read-modify-writes: fibers only switch at barriers;
 *   - async_work_group_copy is carried out by every work-item (each copies
 *     the same values), so wait_group_events has nothing left to wait for;
 *   - native_* and the other built-ins map to the precise libm functions
 *     (the one deliberate deviation, as for the CUDA sources).
 */
#ifndef ADGPU_OCL_SHIM_H
#define ADGPU_OCL_SHIM_H

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <cfloat>
#include <functional>

using std::sqrt; using std::sin; using std::cos; using std::floor; using std::ceil; using std::fabs;
using std::copysign; using std::atan2; using std::exp; using std::fmin; using std::fmax; using std::fmod;
using std::pow; using std::acos;

typedef unsigned int uint;
typedef unsigned short ushort;
typedef unsigned char uchar;

/* ---- address-space and kernel qualifiers ------------------------------- */
#define __kernel
#define __global
#define __constant
#define __private
#define restrict __restrict__

/* ---- vector types ------------------------------------------------------ */
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
static inline float3 make_float3(float x, float y, float z) { float3 r = {x, y, z}; return r; }
static inline float4 make_float4(float x, float y, float z, float w) { float4 r = {x, y, z, w}; return r; }
static inline float4 operator+(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
static inline float4 operator-(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
static inline float4 operator*(float4 a, float4 b) { return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
static inline float4 operator*(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
static inline float4 operator*(float s, float4 a) { return a * s; }
static inline float4 operator/(float4 a, float s) { return make_float4(a.x / s, a.y / s, a.z / s, a.w / s); }
static inline float4 operator-(float4 a) { return make_float4(-a.x, -a.y, -a.z, -a.w); }
static inline float4& operator+=(float4& a, float4 b) { a = a + b; return a; }
static inline float4& operator-=(float4& a, float4 b) { a = a - b; return a; }
static inline float4& operator*=(float4& a, float s) { a = a * s; return a; }
static inline float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
static inline float3 operator*(float s, float3 a) { return a * s; }
static inline float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
static inline float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
static inline float3& operator+=(float3& a, float3 b) { a = a + b; return a; }
static inline float3& operator-=(float3& a, float3 b) { a = a - b; return a; }
static inline float3& operator*=(float3& a, float s) { a = a * s; return a; }

/* geometric built-ins: cross of float4 is the cross of xyz with w = 0 */
static inline float4 cross(float4 a, float4 b)
{
	return make_float4(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x, 0.0f);
}
static inline float3 cross(float3 a, float3 b)
{
	return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float dot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
static inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float length(float4 a) { return sqrtf(dot(a, a)); }
static inline float length(float3 a) { return sqrtf(dot(a, a)); }
static inline float distance(float4 a, float4 b) { return length(a - b); }
static inline float distance(float3 a, float3 b) { return length(a - b); }
static inline float fast_length(float4 a) { return length(a); }
static inline float fast_length(float3 a) { return length(a); }
static inline float fast_distance(float4 a, float4 b) { return distance(a, b); }
static inline float fast_distance(float3 a, float3 b) { return distance(a, b); }
static inline float4 fast_normalize(float4 a) { return a / length(a); }
static inline float3 fast_normalize(float3 a) { return a / length(a); }
static inline float4 normalize(float4 a) { return a / length(a); }
static inline float3 normalize(float3 a) { return a / length(a); }

/* ---- math built-ins (precise host equivalents) ------------------------- */
static inline float native_divide(float a, float b) { return a / b; }
static inline float native_recip(float a) { return 1.0f / a; }
static inline float native_sqrt(float a) { return sqrtf(a); }
static inline float native_rsqrt(float a) { return 1.0f / sqrtf(a); }
static inline float native_sin(float a) { return sinf(a); }
static inline float native_cos(float a) { return cosf(a); }
static inline float native_exp(float a) { return expf(a); }
static inline float native_powr(float a, float b) { return powf(a, b); }
static inline float degrees(float r) { return r * (180.0f / 3.14159265358979323846f); }
static inline float radians(float d) { return d * (3.14159265358979323846f / 180.0f); }

/* ---- work-item coordinates (set by the fiber scheduler) --------------- */
struct uint3_ { unsigned int x, y, z; };      /* as in simt_shim.h */
extern thread_local uint3_ adgpu_sim_threadIdx;
extern thread_local uint3_ adgpu_sim_blockIdx;
extern thread_local uint3_ adgpu_sim_blockDim;
#define get_local_id(d) (adgpu_sim_threadIdx.x)
#define get_group_id(d) (adgpu_sim_blockIdx.x)
#define get_local_size(d) (adgpu_sim_blockDim.x)
#define get_global_id(d) (adgpu_sim_blockIdx.x * adgpu_sim_blockDim.x + adgpu_sim_threadIdx.x)

/* ---- synchronisation ----------------------------------------------------- */
void adgpu_sim_syncthreads();
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2
static inline void barrier(int) { adgpu_sim_syncthreads(); }
static inline void mem_fence(int) {}

typedef int event_t;
template <class T>
static inline event_t async_work_group_copy(T* dst, const T* src, size_t n, event_t)
{
	memcpy((void*)dst, (const void*)src, n * sizeof(T));
	return 0;
}
static inline void wait_group_events(int, event_t*) {}

/* ---- atomics (fibers switch only at barriers) -------------------------- */
static inline int atomic_add(volatile int* p, int v) { int o = *p; *p = o + v; return o; }
static inline int atomic_sub(volatile int* p, int v) { int o = *p; *p = o - v; return o; }
static inline unsigned atomic_add(volatile unsigned* p, unsigned v) { unsigned o = *p; *p = o + v; return o; }
static inline unsigned atomic_cmpxchg(volatile unsigned* p, unsigned cmp, unsigned val)
{
	unsigned o = *p;
	if (o == cmp) *p = val;
	return o;
}
static inline int atomic_cmpxchg(volatile int* p, int cmp, int val)
{
	int o = *p;
	if (o == cmp) *p = val;
	return o;
}

/* ---- launch (simt_shim.cpp) ---------------------------------------------- */
void adgpu_ref_launch(unsigned blocks, unsigned threads, const std::function<void()>& body);

#endif
