// adgpu_device.cuh -- device-side data layout and scorer of the B200 engine.
//
// A pose (one genotype of one ligand) is scored by a "pose group" of TPP
// threads (32: one warp; 64/128: several warps joined by a named barrier).
// Per-ligand constant tables are repacked once on the host (adgpu_tables.cpp)
// into the LigDev layout below; the grid maps are re-laid out so that the 8
// corners of one cell of one map are 32 contiguous, 32-byte-aligned bytes,
// and all maps of a cell sit together (e, d first, then the type maps), so an
// atom's three trilinear lookups are six 128-bit loads from one cell record.
//
// Arithmetic follows the reference scorer operation by operation
// (gpu_calc_energy, cuda/calcenergy.cu:114-453; gpu_calc_energrad,
// cuda/calcMergeEneGra.cu:48-900), including its fixed-point gradient
// accumulation (terms rounded to 1/1024 and clamped to +-8, cuda/GpuData.h:31-35),
// so results agree with the reference to float rounding of single terms.
#pragma once
#include <cstdint>
#include <cfloat>
#include <cuda_runtime.h>

namespace adgpu {

// ---- constants (common/calcenergy_basic.h, common/defines.h, cuda/GpuData.h) ----
constexpr float kDegToRad = 0.0174533f;
constexpr float kPi = 3.14159265358979323846f;
constexpr float kPiTimes2 = 2.0f * kPi;
constexpr float kInvPiTimes2 = 1.0f / kPiTimes2;
constexpr float kTermScale = 1024.0f;
constexpr float kOneOverTermScale = 1.0f / 1024.0f;
constexpr float kMaxTerm = 8192.0f;
// 1.5 * 2^23: a float of magnitude up to 2^22 added to it rounds to an integer
// (nearest, ties to even) and the sum's bits are kRoundBits + that integer
constexpr float kRoundMagic = 12582912.0f;
constexpr uint32_t kRoundBits = 0x4B400000u;
constexpr float kMaxEnergy = FLT_MAX / 100.0f;
constexpr float kInfinitesimalRadian = 1E-3f;
constexpr float kInvInfinitesimalRadian = 1.0f / kInfinitesimalRadian;
constexpr float kScAngstromRadian = 1.0f / (kDegToRad * kDegToRad);
constexpr float kOutOfGridPenalty = 16777216.0f;
constexpr int kOutOfGridForce = 16777216;
constexpr int kMaxAtoms = 256;
constexpr int kMaxGenes = 63;
constexpr int kGenotypeStride = 64;

// ---- repacked per-ligand tables --------------------------------------------------
// Pair record of a pair with other exponents than the AD4 force field's
// (modified pair potentials): the type-pair parameters and the
// charge/desolvation prefactors of one intramolecular contributor, 32 bytes.
struct __align__(16) PairRec {
	float ac, bd, reqm, dsolv_pref;   // VWpars_AC, VWpars_BD, reqm_AB, (S1+qasp|q1|)V2+(S2+qasp|q2|)V1
	float qq;                         // coeff_elec*q1*q2
	float vbond;                      // G for a CG-G0 pair, else 0
	uint32_t ij;                      // atom1 | atom2<<8 | m<<16 | n<<24
	uint32_t pad;
};

// Two pairs of the AD4 force field (exponents m = 12 and n = 6 or 10), the
// ones one thread takes in one step of the pair loop: pair A of an aligned
// group of 32 pairs (one warp instruction) and pair B of the next group,
// 64 bytes in four quads whose fields interleave A and B, so packed FP32x2
// instructions take both pairs' operands straight from the loaded registers:
//   q0 = (AC_A, AC_B, b6_A, b6_B)     VWpars_AC; VWpars_BD of a 12-6 pair, else 0
//   q1 = (b10_A, b10_B, reqm_A, reqm_B)  VWpars_BD of a 12-10 pair, else 0; reqm_AB
//   q2 = (ds_A, ds_B, qq_A, qq_B)     coeff_desolv*((S1+qasp|q1|)V2 + (S2+qasp|q2|)V1); coeff_elec*q1*q2
//   q3 = (G_A, G_B, ij_A, ij_B)       G of a CG-G0 pair, else 0; atom1 | atom2 << 8
// With BD in b6 or b10 by the pair's n (the other 0) the vdW/H-bond energy is
// AC/sd^12 - b6/sd^6 - b10/sd^10 with no select.  The 32 records of a group
// pair are stored quad by quad (quad j of record r at float4 index
// (r/32)*128 + j*32 + r%32), so a warp's load of one quad reads 512
// contiguous bytes.  Padding entries (lists are whole group pairs) have every
// coefficient 0 and both atoms the same: they add exactly 0 to energies and
// forces.
__host__ __device__ inline uint32_t pair2_quad(uint32_t rec, uint32_t j) { return (rec / 32u) * 128u + j * 32u + rec % 32u; }

// Slot (record, half) of the s-th pair of the ordered list of AD4 pairs:
// group s/32 is half (s/32) % 2 of records (s/64)*32 .. +31, lane s % 32.
__host__ __device__ inline void pair2_slot(uint32_t s, uint32_t* rec, uint32_t* half)
{
	*rec = (s / 64u) * 32u + (s % 32u);
	*half = (s / 32u) & 1u;
}
// Records for n ordered AD4 pairs (whole groups of 64 pairs, padded).
__host__ __device__ inline uint32_t pair2_records(uint32_t n) { return (n + 63u) / 64u * 32u; }

// Writes one pair into half h of record rec (quads Q).
__host__ __device__ inline void pair2_set(float4* Q, uint32_t rec, uint32_t h, float ac, float b6, float b10, float reqm,
                                          float ds, float qq, float vb, uint32_t ij)
{
	float* q0 = reinterpret_cast<float*>(Q + pair2_quad(rec, 0));
	float* q1 = reinterpret_cast<float*>(Q + pair2_quad(rec, 1));
	float* q2 = reinterpret_cast<float*>(Q + pair2_quad(rec, 2));
	float* q3 = reinterpret_cast<float*>(Q + pair2_quad(rec, 3));
	q0[h] = ac; q0[2 + h] = b6;
	q1[h] = b10; q1[2 + h] = reqm;
	q2[h] = ds; q2[2 + h] = qq;
	q3[h] = vb; reinterpret_cast<uint32_t*>(q3)[2 + h] = ij;
}
// A padding record (both halves) for lane position rec % 32 of an N-atom
// ligand: the atoms are spread so that padded lanes do not all hit one
// shared-memory bank.
__host__ __device__ inline void pair2_pad(float4* Q, uint32_t rec, uint32_t N)
{
	const uint32_t a = (rec % 32u) % N;
	for (uint32_t h = 0; h < 2; h++) pair2_set(Q, rec, h, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, a | (a << 8));
}

// Stored position of element p of a list of n (torsion items; pairs in the
// kernel-API repack of adgpu_noalloc.cu) in warp-interleaved order.  The reference lists pairs by first atom and items
// by torsion, so 32 consecutive entries mostly share an atom or a torsion and
// a warp's shared-memory gradient atomics on it would serialise.  The list is
// cut into up to 32 consecutive stretches of K entries and stored row by row:
// one warp instruction reads one entry of each stretch.  Sums over the list
// are fixed-point (order-free) or float energies (order within rounding).
__host__ __device__ inline uint32_t interleave_pos(uint32_t p, uint32_t n)
{
	const uint32_t K = (n + 31) / 32;                    // stretch length
	if (K <= 1) return p;
	const uint32_t full = n / K, rem = n - full * K;     // full stretches; length of the last, partial one
	const uint32_t l = p / K, k = p % K;                 // stretch, row
	return k * full + (k < rem ? k : rem) + l;
}

struct LigDev {
	// sizes (npairs: all intramolecular pairs; npairs2: two-pair records of
	// the AD4 pairs; ngpairs: pairs with other exponents)
	int natoms, nlig, ngenes, ntors, npairs, ntoritems;
	int npairs2, ngpairs;
	int coupled;                 // 1: the two pairs of every record share their first atom
	int map_e;                   // index of the e map in the cell record (0)
	// grid
	int gx, gy, gz;              // grid points per axis
	int cells_x, cells_xy;       // cells per row / plane
	int rec_floats;              // floats per cell record = 8*(num_maps)
	float spacing, inv_spacing;
	float coeff_desolv, elec_min_distance, half_smooth;
	// tables (device pointers)
	const float4* atom_xyzq;     // reference coordinates (grid units) + charge
	const uint32_t* atom_info;   // bits 0-7 map-record slot, bit 8 ignore_inter, bit 9 general rotation, bits 16-31 chain start
	const uint8_t* chain_len;    // torsion rotations per atom
	const uint8_t* chain;        // torsion ids, per atom, in application order
	const float4* tors_uv;       // rotatable bond unit vectors
	const float4* tors_mv;       // rotatable bond moving vectors
	const int2* tors_ends;       // rotatable bond atom pair
	const uint32_t* tor_items;   // (torsion<<8 | atom) per rotating atom, grouped by torsion
	const float4* pairs2;        // AD4 pairs, two per record (quads, pair2_quad)
	const PairRec* gpairs;       // pairs with other exponents
	const float* grid;           // cell records, 32-byte aligned
	const int* f3_bias;          // with coupled tables: start value of each atom's fixed-point force components (couple_force); nullptr: 0
};

// ---- math helpers (cuda/calcenergy.cu:31-109) ----------------------------------
__device__ __forceinline__ float fmod_pi2(float x) { return x - (float)(int)(kInvPiTimes2 * x) * kPiTimes2; }

// The reference's acos fit (cuda/calcenergy.cu:48-65); the orientation
// gradient is defined through it, so it is kept term for term.
__device__ __forceinline__ float fast_acos(float cosine)
{
	const float a = 9.78056e-05f, b = -0.00104588f, c = 0.00418716f, d = -0.00314347f;
	const float e = 2.74084f, f = 0.370388f, o = -(a + b + c + d);
	float x = fabsf(cosine);
	float x2 = x * x, x3 = x2 * x, x4 = x3 * x;
	float ac = (((o * x4 + a) * x3 + b) * x2 + c) * x + d
	           + e * sqrtf(2.0f - sqrtf(2.0f + 2.0f * x)) - f * sqrtf(2.0f - 2.0f * x);
	return copysignf(ac, cosine) + (float)(cosine < 0.0f) * kPi;
}

__device__ __forceinline__ float3 cross3(float3 u, float3 v)
{
	return make_float3(u.y * v.z - v.y * u.z, v.x * u.z - u.x * v.z, u.x * v.y - v.x * u.y);
}

__device__ __forceinline__ float4 qmul(float4 a, float4 b)
{
	return make_float4(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
	                   a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
	                   a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w,
	                   a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}

// quaternion_rotate, cuda/calcenergy.cu:95-109
__device__ __forceinline__ float3 qrot(float3 v, float4 q)
{
	float3 qv = make_float3(q.x, q.y, q.z);
	float3 z = cross3(qv, v);
	z.x *= 2.0f; z.y *= 2.0f; z.z *= 2.0f;
	float3 c = cross3(qv, z);
	return make_float3(v.x + z.x * q.w + c.x, v.y + z.y * q.w + c.y, v.z + z.z * q.w + c.z);
}

__device__ __forceinline__ int quant(float v)
{
	return __float2int_rn(fminf(kMaxTerm, fmaxf(-kMaxTerm, kTermScale * v)));
}

// quant() of v / kTermScale: for a value already multiplied by the scale.
__device__ __forceinline__ int quant_scaled(float v)
{
	return __float2int_rn(fminf(kMaxTerm, fmaxf(-kMaxTerm, v)));
}

// ---- PRNG: the reference's per-thread LCG (cuda/auxiliary_genetic.cu:29-79) ------
__device__ __forceinline__ uint32_t lcg_next(uint32_t& s) { s = 1103515245u * s + 12345u; return s; }
__device__ __forceinline__ float lcg_float(uint32_t& s) { return ((float)lcg_next(s) / 4294967296.0f) * 0.999999f; }
__device__ __forceinline__ void map_angle(float& a)
{
	while (a >= 360.0f) a -= 360.0f;
	while (a < 0.0f) a += 360.0f;
}

// ---- pose group ------------------------------------------------------------------
// TPP threads scoring one pose.  TPP == 32 is warp-synchronous; larger groups
// sync with a named barrier (id 1 + group index within the CTA).
template <int TPP>
struct Group {
	int rank;          // 0..TPP-1
	int bar_id;        // named barrier for TPP > 32
	float* red;        // TPP/32 * 8 floats of scratch for cross-warp reductions

	__device__ static constexpr int size() { return TPP; }

	// Barrier ids are immediates so that a kernel reserves only the ids it
	// uses (a register id makes ptxas reserve all 16, which caps resident
	// CTAs per SM at 4).  A 128-thread group is a whole 128-thread CTA.
	__device__ __forceinline__ void sync() const
	{
		if constexpr (TPP == 32) __syncwarp();
		else if constexpr (TPP == 128) __syncthreads();
		else {
			if (bar_id == 1) asm volatile("bar.sync 1, 64;" ::: "memory");
			else asm volatile("bar.sync 2, 64;" ::: "memory");
		}
	}

	__device__ __forceinline__ float sum(float v) const
	{
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
		if constexpr (TPP == 32) {
			return v;
		} else {
			const int w = rank >> 5;
			sync();
			if ((rank & 31) == 0) red[w] = v;
			sync();
			float s = 0.0f;
#pragma unroll
			for (int i = 0; i < TPP / 32; i++) s += red[i];
			return s;
		}
	}

	// K <= 8 sums in one pass, each added in the same order as sum() adds a
	// single value.  scratch_free: the caller has just passed a group barrier
	// after the scratch's last readers, so the leading barrier is skipped.
	// Within a warp the values take sum()'s xor butterfly (partners at lane
	// distance 16, 8, 4, 2, 1) as a reduce-scatter: at distances 16, 8 and 4
	// a lane keeps half of its values and sends its partner the other half,
	// so every partial sum is the one sum() forms, and lanes 4k .. 4k+3 end
	// with value k: 9 shuffles and 9 adds for up to eight values instead of 5
	// of each per value, then (one warp per group) one shuffle per value to
	// hand it to every lane.
	template <int K>
	__device__ __forceinline__ void sum_n(float* v, bool scratch_free = false) const
	{
		static_assert(K >= 1 && K <= 8, "sum_n takes 1 to 8 values");
		constexpr unsigned kAll = 0xffffffffu;
		const int lane = rank & 31;
		const bool h16 = (lane & 16) != 0, h8 = (lane & 8) != 0, h4 = (lane & 4) != 0;
		float w4[4], w2[2];
#pragma unroll
		for (int i = 0; i < 4; i++) {
			const float lo = i < K ? v[i] : 0.0f, hi = 4 + i < K ? v[4 + i] : 0.0f;
			const float keep = h16 ? hi : lo, send = h16 ? lo : hi;
			w4[i] = keep + __shfl_xor_sync(kAll, send, 16);
		}
#pragma unroll
		for (int i = 0; i < 2; i++) {
			const float keep = h8 ? w4[2 + i] : w4[i], send = h8 ? w4[i] : w4[2 + i];
			w2[i] = keep + __shfl_xor_sync(kAll, send, 8);
		}
		float w1;
		{
			const float keep = h4 ? w2[1] : w2[0], send = h4 ? w2[0] : w2[1];
			w1 = keep + __shfl_xor_sync(kAll, send, 4);
		}
		w1 += __shfl_xor_sync(kAll, w1, 2);
		w1 += __shfl_xor_sync(kAll, w1, 1);
		if constexpr (TPP == 32) {
#pragma unroll
			for (int k = 0; k < K; k++) v[k] = __shfl_sync(kAll, w1, 4 * k);
		} else {
			const int w = rank >> 5, mine = lane >> 2;
			if (!scratch_free) sync();
			if ((lane & 3) == 0 && mine < K) red[w * 8 + mine] = w1;
			sync();
#pragma unroll
			for (int k = 0; k < K; k++) {
				float s = 0.0f;
				for (int i = 0; i < TPP / 32; i++) s += red[i * 8 + k];
				v[k] = s;
			}
		}
	}
};

// ---- per-pose shared-memory scratch -------------------------------------------------
// Layout (natoms rounded up to a multiple of 4):
//   tq [ntors] float4; xyz [N] float4 (x, y, z, 0); f3 [3N] int; gg [64] int
// An atom's coordinates are one 16-byte load, so a pair reads both its atoms
// with two shared-memory loads.  Its fixed-point force is f3[3a .. 3a+2]:
// one address per atom for the three components, and since 3 is odd, atoms
// whose indices differ mod 32 fall in different banks, as in three separate
// arrays.
struct PoseSmem {
	float4* xyz;
	int* f3;
	float4* tq;
	float2* gsc;       // sin/cos of theta, phi and half the rotation angle
	int* gg;
};

__host__ __device__ inline int pose_smem_bytes(int natoms, int ntors)
{
	int n4 = (natoms + 3) & ~3;
	return (7 * n4) * 4 + ntors * 16 + 32 + 64 * 4;
}

__device__ __forceinline__ PoseSmem carve_pose(char* base, int natoms, int ntors)
{
	PoseSmem s;
	int n4 = (natoms + 3) & ~3;
	float* f = reinterpret_cast<float*>(base);
	s.tq = reinterpret_cast<float4*>(f);          // 16-byte aligned first
	f += ntors * 4;
	s.gsc = reinterpret_cast<float2*>(f);
	f += 8;
	s.xyz = reinterpret_cast<float4*>(f);         // still 16-byte aligned
	f += 4 * n4;
	s.f3 = reinterpret_cast<int*>(f);
	s.gg = s.f3 + 3 * n4;
	return s;
}

// Genotype-derived general rotation (cuda/calcMergeEneGra.cu:92-120).
struct GenRot {
	float4 q;       // unit quaternion
	float3 mv;      // translation (grid units)
	float sin_theta, sin_half, is_theta_gt_pi;
};

// The general rotation from the sines and cosines step 1 of score_pose left
// in shared memory (sin/cos of theta, phi and half the rotation angle,
// cuda/calcMergeEneGra.cu:92-120).
__device__ __forceinline__ GenRot genrot_from(const float* g, bool has_ligand, const float2* sc)
{
	GenRot r;
	r.q = make_float4(0.f, 0.f, 0.f, 1.f);
	r.mv = make_float3(0.f, 0.f, 0.f);
	r.sin_theta = 0.f; r.sin_half = 0.f; r.is_theta_gt_pi = 1.f;
	if (has_ligand) {
		const float st = sc[0].x, ct = sc[0].y, sp = sc[1].x, cp = sc[1].y, sh = sc[2].x, ch = sc[2].y;
		r.mv = make_float3(g[0], g[1], g[2]);
		r.q = make_float4(sh * st * cp, sh * st * sp, sh * ct, ch);
		r.sin_theta = st; r.sin_half = sh;
		r.is_theta_gt_pi = 1.0f - 2.0f * (float)(st < 0.0f);
	}
	return r;
}

// ---- intramolecular pairs, two per thread with packed FP32 -------------------------
// sm_100 executes FADD2/FMUL2/FFMA2: one instruction on two floats.  The pair
// loop is issue bound, so each thread takes two pairs per step and runs their
// arithmetic packed; compares, reciprocals and the fixed-point atomics stay
// per pair.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2s(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b, exactly (one rounding of -1*b + a)
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) { return __ffma2_rn(f2s(-1.0f), b, a); }
__device__ __forceinline__ float2 f2rcp(float2 a) { return f2(__fdividef(1.0f, a.x), __fdividef(1.0f, a.y)); }
// 1.0f where a < b, else 0.0f (one FSET, no predicate and select)
__device__ __forceinline__ float lt1(float a, float b)
{
	float r;
	asm("set.lt.f32.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
	return r;
}

// inv^e by squaring (the general-exponent path of modified pair potentials)
static __device__ __noinline__ float pow_int(float b, int e)
{
	float r = 1.0f;
	while (e) { if (e & 1) r *= b; b *= b; e >>= 1; }
	return r;
}

// The fixed-point force of one pair (components already scaled by 1024):
// -q on the first atom, +q on the second (f3: three ints per atom).
__device__ __forceinline__ void pair_force(int* f3, uint32_t i, uint32_t j, float gx, float gy, float gz)
{
	const int ix = quant_scaled(gx), iy = quant_scaled(gy), iz = quant_scaled(gz);
	int* fi = f3 + 3 * i;
	int* fj = f3 + 3 * j;
	atomicAdd(fi, -ix); atomicAdd(fi + 1, -iy); atomicAdd(fi + 2, -iz);
	atomicAdd(fj, ix); atomicAdd(fj + 1, iy); atomicAdd(fj + 2, iz);
}

// The fixed-point forces of a couple (pairs A and B sharing atom c, second
// atoms i and j): c's part of the two is summed in registers and added once.
// A component is clamped to +-kMaxTerm like quant_scaled and rounded by one
// packed add of kRoundMagic for both pairs (the same integer as
// __float2int_rn): its bits are kRoundBits + the quantum.  Atoms i and j
// take the bits as they are and c minus both, so each add carries a known
// offset (+kRoundBits for i and j, -2 kRoundBits for c); the integer adds
// wrap, and every atom's forces start at minus the sum of its offsets over
// the ligand's records (L.f3_bias, from the tables), so they end exact.
__device__ __forceinline__ float clamp_term(float v) { return fminf(kMaxTerm, fmaxf(-kMaxTerm, v)); }
__device__ __forceinline__ void couple_force(unsigned* f3, uint32_t c, uint32_t i, uint32_t j, float2 gx, float2 gy, float2 gz)
{
	const float2 mg = f2s(kRoundMagic);
	const float2 rx = f2add(f2(clamp_term(gx.x), clamp_term(gx.y)), mg);
	const float2 ry = f2add(f2(clamp_term(gy.x), clamp_term(gy.y)), mg);
	const float2 rz = f2add(f2(clamp_term(gz.x), clamp_term(gz.y)), mg);
	const unsigned ax = __float_as_uint(rx.x), ay = __float_as_uint(ry.x), az = __float_as_uint(rz.x);
	const unsigned bx = __float_as_uint(rx.y), by = __float_as_uint(ry.y), bz = __float_as_uint(rz.y);
	unsigned* fc = f3 + 3 * c;
	unsigned* fi = f3 + 3 * i;
	unsigned* fj = f3 + 3 * j;
	atomicAdd(fc, 0u - ax - bx); atomicAdd(fc + 1, 0u - ay - by); atomicAdd(fc + 2, 0u - az - bz);
	atomicAdd(fi, ax); atomicAdd(fi + 1, ay); atomicAdd(fi + 2, az);
	atomicAdd(fj, bx); atomicAdd(fj + 1, by); atomicAdd(fj + 2, bz);
}

// Energy of the AD4 pairs this thread takes (records rank, rank + TPP, ...),
// with, for GRAD, their fixed-point forces added to S.f3.  The terms are the
// reference's (cuda/calcMergeEneGra.cu:418-602) rewritten with one reciprocal
// square root and three reciprocals per pair instead of divisions and __powf:
// (AC - sd^(m-n) BD) sd^-m = AC/sd^12 - BD/sd^n; the smoothed distance
// (|reqm - r| >= hs ? r + copysign(hs, reqm - r) : reqm) as reqm clamped to
// [r - hs, r + hs], the elec_min_distance floor as a max (and a min on 1/r).
// TERMS (energy only): also adds this thread's vdW/H-bond, electrostatic,
// desolvation and CG-G0 sums to tsum[0..3].
// With COUPLED (the host's tables, L.coupled) the two pairs of a record share
// their first atom: one position load and one set of atomics for it.
template <int TPP, bool GRAD, bool TERMS, bool COUPLED>
__device__ __forceinline__ float pair_loop(const LigDev& L, const PoseSmem& S, int rank, float* tsum)
{
	// loop invariants read once: when L lives in shared memory (the engine's
	// per-task arguments) the force atomics below would otherwise force a
	// reload of every field in every iteration
	const float hs = L.half_smooth, emd = L.elec_min_distance;
	const float inv_emd = __fdividef(1.0f, emd);
	const int nrec = L.npairs2;
	const float spacing = L.spacing, inv_spacing = L.inv_spacing;
	const float4* const xyz = S.xyz;
	int* const f3 = S.f3;
	float2 esum = f2s(0.0f);
	float2 t_vdw = f2s(0.0f), t_el = f2s(0.0f), t_ds = f2s(0.0f), t_cg = f2s(0.0f);
	// record d = rank + TPP*i: quads at pair2_quad(d, j); the pointer steps
	// TPP/32 blocks of 128 quads per iteration
	const float4* pr = L.pairs2 + (rank / 32) * 128 + (rank % 32);
	for (int d = rank; d < nrec; d += TPP, pr += (TPP / 32) * 128) {
		const float4 q0 = __ldg(pr), q1 = __ldg(pr + 32), q2 = __ldg(pr + 64), q3 = __ldg(pr + 96);
		const uint32_t ija = __float_as_uint(q3.z), ijb = __float_as_uint(q3.w);
		const uint32_t a1 = ija & 0xFFu, a2 = ija >> 8, b1 = COUPLED ? a1 : (ijb & 0xFFu), b2 = ijb >> 8;
		const float4 pa1 = xyz[a1], pa2 = xyz[a2], pb2 = xyz[b2];
		const float4 pb1 = COUPLED ? pa1 : xyz[b1];
		const float2 sx = f2(pa1.x - pa2.x, pb1.x - pb2.x);
		const float2 sy = f2(pa1.y - pa2.y, pb1.y - pb2.y);
		const float2 sz = f2(pa1.z - pa2.z, pb1.z - pb2.z);
		const float2 d2g = f2fma(sz, sz, f2fma(sy, sy, f2mul(sx, sx)));
		// coincident atoms (d2g = 0) get r = 0 from a finite reciprocal
		const float2 inv_dist = f2(rsqrtf(fmaxf(d2g.x, 1e-30f)), rsqrtf(fmaxf(d2g.y, 1e-30f)));
		const float2 r = f2mul(f2mul(d2g, inv_dist), f2s(spacing));
		const float2 vb = f2(q3.x, q3.y);             // G for CG-G0 pairs, else 0
		float2 e = f2mul(vb, r);
		float2 pg = vb;
		if constexpr (TERMS) t_cg = f2add(t_cg, e);
		// vdW / H-bond, cut-off 8 A
		{
			const float2 lo = f2add(r, f2s(-hs)), hi = f2add(r, f2s(hs));
			const float2 sd = f2(fminf(fmaxf(q1.z, lo.x), hi.x), fminf(fmaxf(q1.w, lo.y), hi.y));
			const float2 inv = f2rcp(sd);
			const float2 i2 = f2mul(inv, inv), i4 = f2mul(i2, i2), i6 = f2mul(i4, i2);
			const float2 t12 = f2mul(f2(q0.x, q0.y), f2mul(i6, i6));
			const float2 t6 = f2mul(f2(q0.z, q0.w), i6);
			const float2 t10 = f2mul(f2(q1.x, q1.y), f2mul(i6, i4));
			const float2 ev = f2sub(f2sub(t12, t6), t10);
			// cut-off as a 0/1 factor: the terms are finite for every r (sd >= r - hs)
			const float2 in8 = f2(lt1(r.x, 8.0f), lt1(r.y, 8.0f));
			e = f2fma(in8, ev, e);
			if constexpr (TERMS) t_vdw = f2add(t_vdw, f2mul(in8, ev));
			if (GRAD) {
				// d/dsd: (6 b6/sd^6 + 10 b10/sd^10 - 12 AC/sd^12) / sd
				const float2 gv = f2mul(f2fma(f2s(6.0f), t6, f2fma(f2s(10.0f), t10, f2mul(f2s(-12.0f), t12))), inv);
				pg = f2fma(in8, gv, pg);
			}
		}
		// electrostatics and desolvation, cut-off 20.48 A
		{
			const float2 in20 = f2(lt1(r.x, 20.48f), lt1(r.y, 20.48f));
			const float2 rr = f2(fmaxf(r.x, emd), fmaxf(r.y, emd));
			const float2 ir = f2mul(inv_dist, f2s(inv_spacing));
			const float2 inv_r = f2(fminf(ir.x, inv_emd), fminf(ir.y, inv_emd));
			const float2 d2 = f2mul(rr, rr);
			const float2 num = f2fma(f2mul(f2s(-0.1063f), d2), f2fma(f2s(-0.001947f), d2, f2s(1.0f)), f2s(12.96f));
			const float2 den = f2fma(d2, f2fma(d2, f2fma(f2s(0.000112f), d2, f2s(0.00357f)), f2s(0.4137f)), f2s(12.96f));
			const float2 desolv = f2mul(f2mul(f2(q2.x, q2.y), num), f2rcp(den));
			const float2 rs = f2rcp(f2add(rr, f2s(1.26366f)));
			const float2 rs2 = f2mul(rs, rs);
			const float2 diel = f2fma(f2s(1.10859f), rs2, f2s(0.010358f));
			const float2 es = f2mul(f2(q2.z, q2.w), inv_r);
			const float2 ee = f2fma(diel, es, desolv);
			e = f2fma(in20, ee, e);
			if constexpr (TERMS) {
				t_el = f2add(t_el, f2mul(in20, f2mul(diel, es)));
				t_ds = f2add(t_ds, f2mul(in20, desolv));
			}
			if (GRAD) {
				// es (diel / r + 2.21718 rs^3) + 0.0771605 r desolv
				const float2 ge = f2fma(es, f2fma(inv_r, diel, f2mul(f2mul(f2s(2.21718f), rs2), rs)),
				                        f2mul(f2mul(f2s(0.0771605f), rr), desolv));
				pg = f2fma(f2s(-1.0f), f2mul(in20, ge), pg);
			}
		}
		esum = f2add(esum, e);
		if (GRAD) {
			// fixed-point forces; the 1024 scale folded into gdd (a power of two:
			// the same rounding as quant(sub * gdd))
			const float2 gdd = f2mul(pg, f2mul(inv_dist, f2s(-kTermScale)));
			const float2 gx = f2mul(sx, gdd), gy = f2mul(sy, gdd), gz = f2mul(sz, gdd);
			if constexpr (COUPLED) {
				couple_force(reinterpret_cast<unsigned*>(f3), a1, a2, b2, gx, gy, gz);
			} else {
				pair_force(f3, a1, a2, gx.x, gy.x, gz.x);
				pair_force(f3, b1, b2, gx.y, gy.y, gz.y);
			}
		}
	}
	if constexpr (TERMS) {
		tsum[0] += t_vdw.x + t_vdw.y;
		tsum[1] += t_el.x + t_el.y;
		tsum[2] += t_ds.x + t_ds.y;
		tsum[3] += t_cg.x + t_cg.y;
	}
	return esum.x + esum.y;
}

template <int TPP, bool GRAD, bool TERMS = false>
__device__ __forceinline__ float pair_terms(const LigDev& L, const PoseSmem& S, int rank, float* tsum = nullptr)
{
	return L.coupled ? pair_loop<TPP, GRAD, TERMS, true>(L, S, rank, tsum)
	                 : pair_loop<TPP, GRAD, TERMS, false>(L, S, rank, tsum);
}

// Pairs with other exponents than 12-6 / 12-10 (modified pair potentials;
// the AD4 front end has none), one per thread, the reference's terms with
// sd^-m and sd^-n by repeated squaring.
template <int TPP, bool GRAD, bool TERMS = false>
__device__ __forceinline__ float pair_terms_generic(const LigDev& L, const PoseSmem& S, int rank, float* tsum = nullptr)
{
	const float hs = L.half_smooth, emd = L.elec_min_distance;
	float esum = 0.0f;
	for (int p = rank; p < L.ngpairs; p += TPP) {
		const PairRec P = L.gpairs[p];
		const uint32_t a1 = P.ij & 0xFFu, a2 = (P.ij >> 8) & 0xFFu;
		const int m = (int)((P.ij >> 16) & 0xFFu), n = (int)(P.ij >> 24);
		const float4 p1 = S.xyz[a1], p2 = S.xyz[a2];
		const float sx = p1.x - p2.x, sy = p1.y - p2.y, sz = p1.z - p2.z;
		const float d2g = sx * sx + sy * sy + sz * sz;
		const float inv_dist = rsqrtf(fmaxf(d2g, 1e-30f));
		const float r = d2g * inv_dist * L.spacing;
		float e = P.vbond * r, pg = P.vbond;
		if constexpr (TERMS) tsum[3] += e;
		if (r < 8.0f) {
			const float sd = fminf(fmaxf(P.reqm, r - hs), r + hs);
			const float inv = __fdividef(1.0f, sd);
			const float im = pow_int(inv, m), in_ = pow_int(inv, n);
			const float ev = P.ac * im - P.bd * in_;
			e += ev;
			if constexpr (TERMS) tsum[0] += ev;
			if (GRAD) pg += ((float)n * P.bd * in_ - (float)m * P.ac * im) * inv;
		}
		if (r < 20.48f) {
			const float rr = fmaxf(r, emd);
			const float inv_r = fminf(inv_dist * L.inv_spacing, __fdividef(1.0f, emd));
			const float d2 = rr * rr;
			const float num = (-0.1063f * d2) * (-0.001947f * d2 + 1.0f) + 12.96f;
			const float den = d2 * (d2 * (0.000112f * d2 + 0.00357f) + 0.4137f) + 12.96f;
			const float desolv = P.dsolv_pref * __fdividef(L.coeff_desolv * num, den);
			const float rs = __fdividef(1.0f, rr + 1.26366f);
			const float diel = 1.10859f * rs * rs + 0.010358f;
			const float es = P.qq * inv_r;
			e += diel * es + desolv;
			if constexpr (TERMS) { tsum[1] += diel * es; tsum[2] += desolv; }
			if (GRAD) pg -= es * (inv_r * diel + 2.21718f * rs * rs * rs) + 0.0771605f * rr * desolv;
		}
		esum += e;
		if (GRAD) {
			const float gdd = -pg * inv_dist * kTermScale;
			pair_force(S.f3, a1, a2, sx * gdd, sy * gdd, sz * gdd);
		}
	}
	return esum;
}

// ---- the scorer -----------------------------------------------------------------------
// Scores genotype g (shared memory, read-only here).  Returns the energy (same
// value in every thread of the group).  With GRAD, writes dE/dgene to
// grad[0..ngenes) (shared memory).  Leaves the pose coordinates in S.
// REF_GRID: L.grid is the reference's own layout (4 replicated floats per
// point and map, host/src/processgrid.cpp:244-248) instead of cell records;
// the same 8 corner values are read, from two 16-byte loads per map.
// TERMS (energy only): terms[0..7] (written by rank 0) = intermolecular type
// map, electrostatic and desolvation energies, intramolecular vdW/H-bond,
// electrostatic, desolvation and CG-G0 energies, and the number of atoms
// outside the grid.
template <int TPP, bool GRAD, bool REF_GRID = false, bool TERMS = false>
__device__ float score_pose(const LigDev& L, const float* __restrict__ g, float* __restrict__ grad,
                           const PoseSmem& S, const Group<TPP>& G, float* terms = nullptr)
{
	const int rank = G.rank;
	// 1. torsion quaternions (cuda/calcMergeEneGra.cu:160-175, computed once per
	//    torsion) and the sines/cosines of the general rotation, one sincos
	//    per thread: lanes past the torsions take theta, phi and half the angle
	const bool has_lig = L.nlig > 0;
	const int nsc = L.ntors + (has_lig ? 3 : 0);
	for (int k = rank; k < nsc; k += TPP) {
		const int j = k - L.ntors;
		const float ang = j < 0 ? g[6 + k] * kDegToRad * 0.5f
		                        : (j == 0 ? g[4] * kDegToRad : (j == 1 ? g[3] * kDegToRad : g[5] * kDegToRad * 0.5f));
		float s, c;
		sincosf(ang, &s, &c);
		if (j < 0) {
			float4 u = L.tors_uv[k];
			S.tq[k] = make_float4(s * u.x, s * u.y, s * u.z, c);
		} else {
			S.gsc[j] = make_float2(s, c);
		}
	}
	if (GRAD)
		for (int k = rank; k < L.ngenes; k += TPP) S.gg[k] = 0;
	G.sync();
	const GenRot gr = genrot_from(g, has_lig, S.gsc);

	// 2. pose: each atom applies its own torsion chain, then the general rotation
	//    (the per-atom order the reference's rotation list encodes, cuda/calcMergeEneGra.cu:131-190);
	//    the same thread then takes the atom's intermolecular terms (3.)
	float e_acc = 0.0f;
	float tt[TERMS ? 8 : 1] = {0.f};   // TERMS partial sums
	for (int a = rank; a < L.natoms; a += TPP) {
		float4 r4 = L.atom_xyzq[a];
		float3 p = make_float3(r4.x, r4.y, r4.z);
		uint32_t info = L.atom_info[a];
		int cs = info >> 16, cl = L.chain_len[a];
		for (int i = 0; i < cl; i++) {
			int k = L.chain[cs + i];
			float4 m4 = L.tors_mv[k];
			float3 m = make_float3(m4.x, m4.y, m4.z);
			p.x -= m.x; p.y -= m.y; p.z -= m.z;
			p = qrot(p, S.tq[k]);
			p.x += m.x; p.y += m.y; p.z += m.z;
		}
		if ((info & 0x200u) && a < L.nlig) {
			p = qrot(p, gr.q);
			p.x += gr.mv.x; p.y += gr.mv.y; p.z += gr.mv.z;
		}
		S.xyz[a] = make_float4(p.x, p.y, p.z, 0.0f);

		// 3. intermolecular: trilinear interpolation of the type, e and d maps
		//    (cuda/calcMergeEneGra.cu:195-413)
		int fx = 0, fy = 0, fz = 0;
		if (!(info & 0x100u)) {
			float x = p.x, y = p.y, z = p.z;
			float q = r4.w;
			if (x < 0.f || y < 0.f || z < 0.f || x >= (float)(L.gx - 1) || y >= (float)(L.gy - 1) || z >= (float)(L.gz - 1)) {
				e_acc += kOutOfGridPenalty;
				fx = fy = fz = kOutOfGridForce;
				if constexpr (TERMS) tt[7] += 1.0f;
			} else {
				float xl = floorf(x), yl = floorf(y), zl = floorf(z);
				float dx = x - xl, omdx = 1.0f - dx, dy = y - yl, omdy = 1.0f - dy, dz = z - zl, omdz = 1.0f - dz;
				float w0 = omdx * omdy * omdz, w1 = omdx * dy * omdz, w2 = omdx * omdy * dz, w3 = omdx * dy * dz;
				float w4 = dx * omdy * omdz, w5 = dx * dy * omdz, w6 = dx * omdy * dz, w7 = dx * dy * dz;
				int slot = info & 0xFFu;
				float4 t0, t1, e0, e1, d0, d1;
				if constexpr (REF_GRID) {
					const size_t g3 = (size_t)L.gx * L.gy * L.gz;
					const size_t p = (size_t)xl + (size_t)yl * L.gx + (size_t)zl * L.gx * L.gy;
					const size_t M = (size_t)(L.rec_floats / 8 - 2);
					const float4* tp = reinterpret_cast<const float4*>(L.grid + ((((size_t)slot - 2) * g3 + p) << 2));
					const float4* ep = reinterpret_cast<const float4*>(L.grid + ((M * g3 + p) << 2));
					const float4* dp = reinterpret_cast<const float4*>(L.grid + (((M + 1) * g3 + p) << 2));
					t0 = __ldg(tp); t1 = __ldg(tp + 1); e0 = __ldg(ep); e1 = __ldg(ep + 1); d0 = __ldg(dp); d1 = __ldg(dp + 1);
				} else {
					int cell = (int)xl + (int)yl * L.cells_x + (int)zl * L.cells_xy;
					const float4* rec = reinterpret_cast<const float4*>(L.grid + (size_t)cell * L.rec_floats);
					t0 = __ldg(rec + 2 * slot); t1 = __ldg(rec + 2 * slot + 1);
					e0 = __ldg(rec + 0); e1 = __ldg(rec + 1);
					d0 = __ldg(rec + 2); d1 = __ldg(rec + 3);
				}
				float vt = t0.x * w0 + t0.y * w1 + t0.z * w2 + t0.w * w3 + t1.x * w4 + t1.y * w5 + t1.z * w6 + t1.w * w7;
				float ve = e0.x * w0 + e0.y * w1 + e0.z * w2 + e0.w * w3 + e1.x * w4 + e1.y * w5 + e1.z * w6 + e1.w * w7;
				float vd = d0.x * w0 + d0.y * w1 + d0.z * w2 + d0.w * w3 + d1.x * w4 + d1.y * w5 + d1.z * w6 + d1.w * w7;
				e_acc += vt;
				e_acc += q * ve;
				e_acc += fabsf(q) * vd;
				if constexpr (TERMS) { tt[0] += vt; tt[1] += q * ve; tt[2] += fabsf(q) * vd; }
				if (GRAD) {
					// corners: .x .y .z .w of rec0 = 000 010 001 011 ; of rec1 = 100 110 101 111
#define ADGPU_GX(c0, c1) (omdz * (omdy * (c1.x - c0.x) + dy * (c1.y - c0.y)) + dz * (omdy * (c1.z - c0.z) + dy * (c1.w - c0.w)))
#define ADGPU_GY(c0, c1) (omdz * (omdx * (c0.y - c0.x) + dx * (c1.y - c1.x)) + dz * (omdx * (c0.w - c0.z) + dx * (c1.w - c1.z)))
#define ADGPU_GZ(c0, c1) (omdy * (omdx * (c0.z - c0.x) + dx * (c1.z - c1.x)) + dy * (omdx * (c0.w - c0.y) + dx * (c1.w - c1.y)))
					float inv = L.inv_spacing;
					float gxx = ADGPU_GX(t0, t1) * inv, gyy = ADGPU_GY(t0, t1) * inv, gzz = ADGPU_GZ(t0, t1) * inv;
					float q1 = q * inv;
					gxx += q1 * ADGPU_GX(e0, e1); gyy += q1 * ADGPU_GY(e0, e1); gzz += q1 * ADGPU_GZ(e0, e1);
					q1 = fabsf(q1);
					gxx += q1 * ADGPU_GX(d0, d1); gyy += q1 * ADGPU_GY(d0, d1); gzz += q1 * ADGPU_GZ(d0, d1);
#undef ADGPU_GX
#undef ADGPU_GY
#undef ADGPU_GZ
					fx = quant(gxx); fy = quant(gyy); fz = quant(gzz);
				}
			}
		}
		if (GRAD) {
			// the start value that cancels couple_force's rounding offsets
			const unsigned fb = L.f3_bias ? (unsigned)__ldg(L.f3_bias + a) : 0u;
			int* fa = S.f3 + 3 * a;
			fa[0] = (int)((unsigned)fx + fb); fa[1] = (int)((unsigned)fy + fb); fa[2] = (int)((unsigned)fz + fb);
		}
	}
	G.sync();

	// 4. intramolecular pairs (cuda/calcMergeEneGra.cu:418-602)
	if constexpr (TERMS) e_acc += pair_terms<TPP, GRAD, TERMS>(L, S, rank, tt + 3);
	else e_acc += pair_terms<TPP, GRAD>(L, S, rank);
	if (L.ngpairs > 0) {
		if constexpr (TERMS) e_acc += pair_terms_generic<TPP, GRAD, TERMS>(L, S, rank, tt + 3);
		else e_acc += pair_terms_generic<TPP, GRAD>(L, S, rank);
	}
	if constexpr (TERMS) {
		G.template sum_n<8>(tt);
		if (rank == 0)
			for (int k = 0; k < 8; k++) terms[k] = tt[k];
	}
	if (!GRAD) return G.sum(e_acc);
	G.sync();   // every pair's forces are in S.f3

	// 5. torque and total force over the ligand atoms (cuda/calcMergeEneGra.cu:608-661);
	//    the energy rides along as a seventh sum (one cross-warp exchange, not two)
	// sizes and pointers of the steps below read once (when L lives in shared
	// memory, the engine's per-task arguments, the stores to S would otherwise
	// force reloads in every iteration); not held across the pair loop, whose
	// register peak would spill
	const int nlig = L.nlig;
	const float spacing = L.spacing;
	float red[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, e_acc};
	for (int a = rank; a < nlig; a += TPP) {
		const float4 pa = S.xyz[a];
		float3 r = make_float3((pa.x - gr.mv.x) * spacing, (pa.y - gr.mv.y) * spacing, (pa.z - gr.mv.z) * spacing);
		const int* fa = S.f3 + 3 * a;
		float3 f = make_float3(kOneOverTermScale * (float)fa[0], kOneOverTermScale * (float)fa[1], kOneOverTermScale * (float)fa[2]);
		red[3] += f.x; red[4] += f.y; red[5] += f.z;
		float3 t = cross3(r, f);
		red[0] += t.x; red[1] += t.y; red[2] += t.z;
	}
	G.template sum_n<7>(red, true);
	const float energy = red[6];
	if (rank < 3 && nlig > 0) {
		// translation (:676-689) and orientation (:695-815) genes: lane j takes
		// orientation gene 3 + j (phi, theta, rotation angle) with the same code
		// on its own angle, and lane 0 also the translation genes; every gene
		// gets the reference's operations in the reference's order
		if (rank == 0) {
			S.gg[0] = quant(red[3] * spacing);
			S.gg[1] = quant(red[4] * spacing);
			S.gg[2] = quant(red[5] * spacing);
		}
		float tl = norm3df(red[0], red[1], red[2]);
		float oscale = (tl < kInfinitesimalRadian) ? 1.0f : tl * kInvInfinitesimalRadian;
		// sin/cos of half the infinitesimal rotation (SIN/COS_HALF_INFINITESIMAL_RADIAN,
		// common/calcenergy_basic.h:79-80), rounded to float: sin(0.0005) rounds
		// to 0.0005f, cos(0.0005) to 1 - 2^-23
		constexpr float kSinHalfInf = 0x1.0624dep-11f, kCosHalfInf = 0x1.fffffcp-1f;
		float tscale = (tl < kInfinitesimalRadian) ? 0.5f - tl * tl / 48.0f : kSinHalfInf / tl;
		float4 qt = make_float4(red[0] * tscale, red[1] * tscale, red[2] * tscale,
		                        (tl < kInfinitesimalRadian) ? 1.0f - tl * tl * 0.125f : kCosHalfInf);
		float4 tgt = qmul(qt, gr.q);
		// target angle: phi = atan2, theta = 2 pi + sign * acos(z / sin_ang),
		// rotation = 2 acos(w)
		float target;
		if (rank == 0) {
			target = fmod_pi2(atan2f(gr.is_theta_gt_pi * tgt.y, gr.is_theta_gt_pi * tgt.x) + kPiTimes2);
		} else {
			const float sin_ang = sqrtf(1.0f - tgt.w * tgt.w);
			const float ac = fast_acos(rank == 1 ? tgt.z / sin_ang : tgt.w);
			target = rank == 1 ? kPiTimes2 + gr.is_theta_gt_pi * ac : 2.0f * ac;
		}
		const float cur = fmod_pi2(kPiTimes2 + g[3 + rank] * kDegToRad);
		float v = oscale * (fmod_pi2(target - cur + kPi) - kPi);
		const float corr = 4.0f * gr.sin_half * gr.sin_half;
		if (rank == 0) v = v * gr.sin_theta * gr.sin_theta;
		if (rank <= 1) v = v * corr;
		S.gg[3 + rank] = quant(v * kDegToRad);
	}

	// 6. torsion genes: axis . (r x F) summed over each torsion's rotating atoms (:819-880)
	const uint32_t* const tor_items = L.tor_items;
	const int2* const tors_ends = L.tors_ends;
	const int ntoritems = L.ntoritems, ngenes = L.ngenes;
	for (int it = rank; it < ntoritems; it += TPP) {
		uint32_t item = tor_items[it];
		int k = item >> 8, la = item & 0xFF;
		int2 ends = tors_ends[k];
		const float4 e0 = S.xyz[ends.x], e1 = S.xyz[ends.y], pl = S.xyz[la];
		float rx = e0.x, ry = e0.y, rz = e0.z;
		float ux = e1.x - rx, uy = e1.y - ry, uz = e1.z - rz;
		float l = rnorm3df(ux, uy, uz);
		ux *= l; uy *= l; uz *= l;
		float3 r = make_float3(pl.x - rx, pl.y - ry, pl.z - rz);
		const int* fl = S.f3 + 3 * la;
		float3 f = make_float3(kOneOverTermScale * (float)fl[0], kOneOverTermScale * (float)fl[1], kOneOverTermScale * (float)fl[2]);
		float3 t = cross3(r, f);
		float on_axis = (ux * t.x + uy * t.y + uz * t.z) * spacing;
		atomicAdd(&S.gg[6 + k], quant(on_axis * kDegToRad));
	}
	G.sync();
	// 7. fixed point -> float, Angstrom/radian scaling of genes >= 3 (:883-899)
	const float sc = spacing * spacing * kScAngstromRadian;
	for (int k = rank; k < ngenes; k += TPP) {
		float v = kOneOverTermScale * (float)S.gg[k];
		grad[k] = (k >= 3) ? v * sc : v;
	}
	G.sync();
	return energy;
}

}  // namespace adgpu
