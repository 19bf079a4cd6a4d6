// adgpu_kernels.cuh -- the LGA hot-path kernels: GA generation, Solis-Wets,
// ADADELTA, ADAM, FIRE, initial-population scoring, per-run eval sums.
//
// Each reference "block" (one entity of one run) is processed by one pose
// group of TPP threads; a persistent grid of pose groups strides over the
// reference's block indices, so the launch shape no longer depends on the
// entity count.  The reference's per-thread PRNG layout is preserved: a draw
// that the reference makes in thread `lane` of block `b` uses state
// prng[b * ref_threads + lane] here too (cuda/auxiliary_genetic.cu:37), so
// given the same states the same random decisions are taken.
#pragma once
#include "adgpu_device.cuh"
#include "../../include/adgpu_b200.h"

namespace adgpu {

enum LsMethod { LS_SW = 0, LS_AD = 1, LS_ADAM = 2, LS_FIRE = 3 };

// Everything one launch needs, passed by value (kernel parameter space).
struct KArgs {
	LigDev L;
	adgpu_dockpars dp;
	const float* conf_cur;      // GA: current population
	const float* e_cur;
	float* conf;                // GA: next population; LS/initpop: population worked on
	float* e;
	uint32_t* prng;
	int* evals_new;
	int* evals_runs;
	uint32_t nblocks;           // reference blocks (entities) in this launch
	uint32_t ref_threads;       // reference block size (PRNG layout)
	const int* stop_flag;       // nullable: when *stop_flag != 0 the launch does nothing
	unsigned int* work_counter; // nullable: zeroed before the launch; pose groups take blocks from it
};

// The population buffers a block reads and writes: the launch's own
// (bufs_of) or, in the pipelined docking loop, those of the block's
// generation.  Passed apart from KArgs so that KArgs can stay a kernel
// parameter read with constant offsets in the scorer.
struct PopBufs {
	const float* conf_cur;      // GA: current population
	const float* e_cur;
	float* conf;                // GA: next population; LS/initpop: population worked on
	float* e;
};

__device__ __forceinline__ PopBufs bufs_of(const KArgs& a) { return PopBufs{a.conf_cur, a.e_cur, a.conf, a.e}; }

// Per-group scratch carved from dynamic shared memory.
struct GroupSmem {
	PoseSmem pose;
	float* gen; float* best; float* grad; float* s1; float* s2; float* s3; float* s4; float* s5;
	uint32_t* st;     // PRNG states of the reference lanes of this block (GA, SW)
	float* red;       // cross-warp reduction scratch
	int* misc;        // small ints (entity ids, crossover points, ...)
	float* miscf;     // small floats (random numbers, energies)
};

// Shared-memory carveout (percent of the SM's maximum) that lets `ctas` CTAs
// of `bytes` dynamic shared memory each be resident at once; the rest of the
// unified L1/shared array stays L1 cache for the ligand tables and the maps.
// (With no preference the driver picked a 100 KB split: 4 engine CTAs per SM.)
inline int smem_carveout_pct(int bytes, int ctas)
{
	int dev = 0, max_sm = 0;
	if (cudaGetDevice(&dev) != cudaSuccess ||
	    cudaDeviceGetAttribute(&max_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess || max_sm <= 0)
		return -1;
	const long need = (long)ctas * (bytes + 1024);
	const long pct = (need * 100 + max_sm - 1) / max_sm;
	return (int)(pct > 100 ? 100 : pct);
}

__host__ __device__ inline int group_smem_bytes(int natoms, int ntors, int ref_threads, int tpp)
{
	int b = pose_smem_bytes(natoms, ntors);
	b += 8 * 64 * 4;                       // gene arrays
	b += ((ref_threads + 3) & ~3) * 4;     // PRNG states
	b += (tpp / 32) * 8 * 4;               // reduction scratch
	b += 16 * 4 + 16 * 4;                  // misc ints, floats
	return (b + 15) & ~15;
}

__device__ __forceinline__ GroupSmem carve_group(char* base, int natoms, int ntors, int ref_threads, int tpp)
{
	GroupSmem s;
	s.pose = carve_pose(base, natoms, ntors);
	float* f = reinterpret_cast<float*>(base + pose_smem_bytes(natoms, ntors));
	s.gen = f; s.best = f + 64; s.grad = f + 128; s.s1 = f + 192; s.s2 = f + 256; s.s3 = f + 320; s.s4 = f + 384; s.s5 = f + 448;
	f += 512;
	s.st = reinterpret_cast<uint32_t*>(f);
	f += (ref_threads + 3) & ~3;
	s.red = f;
	f += (tpp / 32) * 8;
	s.misc = reinterpret_cast<int*>(f);
	s.miscf = f + 16;
	return s;
}

// The group of this thread and its scratch.
template <int TPP>
__device__ __forceinline__ void group_of(const KArgs& a, int& gid, int& ngroups, Group<TPP>& G, GroupSmem& S)
{
	extern __shared__ __align__(16) char smem[];
	const int gpc = blockDim.x / TPP;               // groups per CTA
	const int local = threadIdx.x / TPP;
	gid = blockIdx.x * gpc + local;
	ngroups = gridDim.x * gpc;
	const int bytes = group_smem_bytes(a.L.natoms, a.L.ntors, (int)a.ref_threads, TPP);
	S = carve_group(smem + local * bytes, a.L.natoms, a.L.ntors, (int)a.ref_threads, TPP);
	G.rank = threadIdx.x % TPP;
	G.bar_id = 1 + local;
	G.red = S.red;
}

// LS entity choice shared by every local search (e.g. cuda/kernel_ad.cu:116-127):
// entity 0 (the elite) is searched only with probability lsearch_rate %.
template <int TPP>
__device__ __forceinline__ int ls_entity(const KArgs& a, uint32_t b, const Group<TPP>& G, const GroupSmem& S)
{
	int ent = (int)(b % a.dp.num_of_lsentities);
	if (ent == 0) {
		if (G.rank == 0) {
			uint32_t s = a.prng[b * a.ref_threads];
			if (100.0f * lcg_float(s) > a.dp.lsearch_rate) ent = (int)a.dp.num_of_lsentities;
			a.prng[b * a.ref_threads] = s;
			S.misc[0] = ent;
		}
		G.sync();
		ent = S.misc[0];
		G.sync();
	}
	return ent;
}

// ---------------------------------------------------------------------------
// ADADELTA (cuda/kernel_ad.cu:60-393): rho 0.8, eps 1e-2, stop when the
// success/fail step-size proxy falls to 0.01 or after max_num_of_iters.
// ADAM (cuda/kernel_adam.cu:55-396): bias-corrected, always max_num_of_iters.
// ---------------------------------------------------------------------------
template <int TPP, int METHOD>
__device__ void gradient_ls_block(const KArgs& a, const PopBufs& pb, uint32_t b, const Group<TPP>& G, const GroupSmem& S)
{
	const int P = a.dp.pop_size, NG = a.dp.num_of_genes;
	const int run = (int)(b / a.dp.num_of_lsentities);
	const int ent = ls_entity<TPP>(a, b, G, S);
	const size_t idx = (size_t)run * P + ent;
	const float* src = pb.conf + idx * kGenotypeStride;
	for (int k = G.rank; k < NG; k += TPP) {
		S.gen[k] = src[k]; S.best[k] = S.gen[k]; S.grad[k] = 0.f; S.s1[k] = 0.f; S.s2[k] = 0.f;
	}
	G.sync();
	float best_e = INFINITY, rho = 1.0f;
	int succ = 0, fail = 0;
	uint32_t it = 0;
	const float RHO = 0.8f, EPS = 1e-2f;
	// ADAM's bias corrections 1 - beta^(it+1): every 32 iterations each lane
	// computes those of iteration it + lane (the same powf of the same
	// arguments), and iteration it takes them from lane it % 32, so the
	// warp runs one powf pair per 32 iterations instead of one per iteration
	float b1r = 0.f, b2r = 0.f;
	do {
		if (METHOD == LS_ADAM && (it & 31u) == 0) {
			const float t = 1.0f + (float)(it + (uint32_t)(G.rank & 31));
			b1r = 1.0f - powf(a.dp.adam_beta1, t);
			b2r = 1.0f - powf(a.dp.adam_beta2, t);
		}
		const float energy = score_pose<TPP, true>(a.L, S.gen, S.grad, S.pose, G);
		float b1p = 0.f, b2p = 0.f;
		if (METHOD == LS_ADAM) {
			b1p = __shfl_sync(0xffffffffu, b1r, (int)(it & 31u));
			b2p = __shfl_sync(0xffffffffu, b2r, (int)(it & 31u));
		}
		for (int k = G.rank; k < NG; k += TPP) {
			float g = S.grad[k];
			if (energy < best_e) S.best[k] = S.gen[k];
			if (METHOD == LS_AD) {
				float sg = RHO * S.s1[k] + (1.0f - RHO) * g * g;
				float delta = -1.0f * g * sqrtf((S.s2[k] + EPS) / (sg + EPS));
				S.s1[k] = sg;
				S.s2[k] = RHO * S.s2[k] + (1.0f - RHO) * delta * delta;
				S.gen[k] += delta;
			} else {
				float mt = a.dp.adam_beta1 * S.s1[k] + (1.0f - a.dp.adam_beta1) * g;
				float vt = a.dp.adam_beta2 * S.s2[k] + (1.0f - a.dp.adam_beta2) * g * g;
				S.s1[k] = mt; S.s2[k] = vt;
				float mp = mt / b1p, vp = vt / b2p;
				S.gen[k] -= mp / (sqrtf(vp) + a.dp.adam_epsilon);
			}
		}
		it++;
		if (METHOD == LS_AD) {
			if (energy < best_e) { best_e = energy; succ++; fail = 0; }
			else { succ = 0; fail++; }
			if (succ >= 4) { rho *= 2.0f; succ = 0; }
			else if (fail >= 4) { rho *= 0.5f; fail = 0; }
		} else {
			if (energy < best_e) best_e = energy;
		}
		G.sync();
	} while (it < a.dp.max_num_of_iters && (METHOD == LS_ADAM || rho > 0.01f));
	float* dst = pb.conf + idx * kGenotypeStride;
	for (int k = G.rank; k < NG; k += TPP) {
		float v = S.best[k];
		if (k >= 3) map_angle(v);
		dst[k] = v;
	}
	if (G.rank == 0) {
		a.evals_new[idx] += (int)it;
		pb.e[idx] = best_e;
	}
	G.sync();
}

// ---------------------------------------------------------------------------
// FIRE (device/kernel_fire.cl:76-895): N_min 5, f_inc 1.2, f_dec 0.8,
// alpha0 0.2, f_alpha 0.99, dt_max 10, dt0 = dt_max/3, stop at dt < 1e-6.
// ---------------------------------------------------------------------------
template <int TPP>
__device__ void fire_block(const KArgs& a, const PopBufs& pb, uint32_t b, const Group<TPP>& G, const GroupSmem& S)
{
	const float DT_INC = 1.2f, DT_DEC = 0.8f, ALPHA_START = 0.2f, ALPHA_DEC = 0.99f, DT_MAX = 10.0f, DT_MIN = 1e-6f;
	const int P = a.dp.pop_size, NG = a.dp.num_of_genes;
	const int run = (int)(b / a.dp.num_of_lsentities);
	const int ent = ls_entity<TPP>(a, b, G, S);
	const size_t idx = (size_t)run * P + ent;
	const float* src = pb.conf + idx * kGenotypeStride;
	float* gen = S.gen; float* best = S.best; float* grad = S.grad;
	float* cgen = S.s1; float* cgrad = S.s2; float* vel = S.s3;
	for (int k = G.rank; k < NG; k += TPP) { gen[k] = src[k]; best[k] = gen[k]; }
	G.sync();
	float energy = pb.e[idx];
	// initial gradient (the OpenCL kernel's gradient-only call, taken from the merged scorer)
	score_pose<TPP, true>(a.L, gen, grad, S.pose, G);
	auto sumsq = [&](const float* v) {
		float s = 0.f;
		for (int k = G.rank; k < NG; k += TPP) s += v[k] * v[k];
		return G.sum(s);
	};
	float alpha = ALPHA_START, dt = DT_MAX / 3.0f;
	uint32_t count_success = 0, it = 0;
	float inv = ALPHA_START * (1.0f / sqrtf(sumsq(grad)));
	for (int k = G.rank; k < NG; k += TPP) vel[k] = -grad[k] * inv;
	float best_e = energy;
	G.sync();
	do {
		for (int k = G.rank; k < NG; k += TPP) cgen[k] = gen[k] + dt * vel[k];
		G.sync();
		const float ce = score_pose<TPP, true>(a.L, cgen, cgrad, S.pose, G);
		float pw = 0.f;
		for (int k = G.rank; k < NG; k += TPP) pw += -cgrad[k] * vel[k];
		const float power = G.sum(pw);
		if (power < 0.0f) {
			inv = ALPHA_START * (1.0f / sqrtf(sumsq(grad)));
			for (int k = G.rank; k < NG; k += TPP) vel[k] = -grad[k] * inv;
			count_success = 0;
			alpha = ALPHA_START;
			dt = dt * DT_DEC;
		} else {
			count_success++;
			if (count_success > 5) { dt = fminf(dt * DT_INC, DT_MAX); alpha = alpha * ALPHA_DEC; }
		}
		G.sync();
		energy = ce;
		for (int k = G.rank; k < NG; k += TPP) { gen[k] = cgen[k]; grad[k] = cgrad[k]; }
		G.sync();
		const float inv_gn = 1.0f / sqrtf(sumsq(grad));
		const float vn = sqrtf(sumsq(vel));
		const float vdg = alpha * vn * inv_gn;
		for (int k = G.rank; k < NG; k += TPP) vel[k] = (1.0f - alpha) * vel[k] - grad[k] * vdg;
		it++;
		if (energy < best_e) {
			best_e = energy;
			for (int k = G.rank; k < NG; k += TPP) best[k] = gen[k];
		}
		G.sync();
	} while (it < a.dp.max_num_of_iters && dt > DT_MIN);
	float* dst = pb.conf + idx * kGenotypeStride;
	for (int k = G.rank; k < NG; k += TPP) {
		float v = best[k];
		if (k >= 3) map_angle(v);
		dst[k] = v;
	}
	if (G.rank == 0) { a.evals_new[idx] += (int)it; pb.e[idx] = best_e; }
	G.sync();
}

// ---------------------------------------------------------------------------
// Solis-Wets with SWAT3 step scaling (cuda/kernel3.cu:30-308).
// ---------------------------------------------------------------------------
template <int TPP>
__device__ void sw_block(const KArgs& a, const PopBufs& pb, uint32_t b, const Group<TPP>& G, const GroupSmem& S)
{
	const int P = a.dp.pop_size, NG = a.dp.num_of_genes;
	const uint32_t T = a.ref_threads;
	const int run = (int)(b / a.dp.num_of_lsentities);
	const int ent = ls_entity<TPP>(a, b, G, S);
	const size_t idx = (size_t)run * P + ent;
	float* gen = S.gen; float* cand = S.s1; float* dev = S.s2; float* bias = S.s3;
	const float* src = pb.conf + idx * kGenotypeStride;
	for (int k = G.rank; k < NG; k += TPP) { gen[k] = src[k]; cand[k] = gen[k]; bias[k] = 0.f; dev[k] = 0.f; }
	for (uint32_t r = G.rank; r < T; r += TPP) S.st[r] = a.prng[b * T + r];
	G.sync();
	const int gs = (a.dp.true_ligand_atoms == 0) * 6;
	const float lig_scale = 1.0f / sqrtf((float)a.dp.num_of_atoms);
	const float gene_scale = 1.0f / sqrtf((float)NG);
	float cur_e = pb.e[idx], rho = 1.0f;
	int succ = 0, fail = 0, iters = 0, evals = 0;
	while (iters < (int)a.dp.max_num_of_iters && rho > a.dp.rho_lower_bound) {
		// reference lane r owns genes gs + r, gs + r + T, ... (its own LCG stream)
		for (uint32_t r = G.rank; r < T; r += TPP) {
			uint32_t s = S.st[r];
			for (int g = gs + (int)r; g < NG; g += (int)T) {
				float r1 = lcg_float(s);
				float r2 = lcg_float(s);
				float d = rho * (2.0f * r1 - 1.0f) * (float)(r2 < gene_scale);
				if (g < 3) d *= a.dp.base_dmov_mul_sqrt3;
				else if (g < 6) d *= a.dp.base_dang_mul_sqrt3 * lig_scale;
				else d *= a.dp.base_dang_mul_sqrt3 * gene_scale;
				dev[g] = d;
			}
			S.st[r] = s;
		}
		G.sync();
		for (int k = gs + G.rank; k < NG; k += TPP) cand[k] = gen[k] + dev[k] + bias[k];
		G.sync();
		float ce = score_pose<TPP, false>(a.L, cand, nullptr, S.pose, G);
		evals++;
		if (ce < cur_e) {
			for (int k = gs + G.rank; k < NG; k += TPP) { gen[k] = cand[k]; bias[k] = 0.6f * bias[k] + 0.4f * dev[k]; }
			cur_e = ce; succ++; fail = 0;
		} else {
			for (int k = gs + G.rank; k < NG; k += TPP) cand[k] = gen[k] - dev[k] - bias[k];
			G.sync();
			ce = score_pose<TPP, false>(a.L, cand, nullptr, S.pose, G);
			evals++;
			if (ce < cur_e) {
				for (int k = gs + G.rank; k < NG; k += TPP) { gen[k] = cand[k]; bias[k] = 0.6f * bias[k] - 0.4f * dev[k]; }
				cur_e = ce; succ++; fail = 0;
			} else {
				for (int k = gs + G.rank; k < NG; k += TPP) bias[k] = 0.5f * bias[k];
				succ = 0; fail++;
			}
		}
		iters++;
		if (succ >= (int)a.dp.cons_limit) { rho *= 2.0f; succ = 0; }
		else if (fail >= (int)a.dp.cons_limit) { rho *= 0.5f; fail = 0; }
		G.sync();
	}
	float* dst = pb.conf + idx * kGenotypeStride;
	for (int k = gs + G.rank; k < NG; k += TPP) {
		float v = gen[k];
		if (k >= 3) map_angle(v);
		dst[k] = v;
	}
	for (uint32_t r = G.rank; r < T; r += TPP) a.prng[b * T + r] = S.st[r];
	if (G.rank == 0) { a.evals_new[idx] += evals; pb.e[idx] = cur_e; }
	G.sync();
}

// ---------------------------------------------------------------------------
// GA generation (cuda/kernel4.cu:28-304): elitism in block run*P, otherwise
// 2 binary tournaments, 2-point crossover, mutation, and scoring.
// ---------------------------------------------------------------------------

// One WARPMINIMUMEXCHANGE network (cuda/kernels.cu:47-64) across a warp.
__device__ __forceinline__ void warp_minimum2(int lane, float& v, int& k)
{
#pragma unroll
	for (int mask = 1; mask < 32; mask <<= 1) {
		int o = lane ^ mask;
		float v2 = __shfl_sync(0xffffffffu, v, o);
		int k2 = __shfl_sync(0xffffffffu, k, o);
		int flag = ((v < v2) ^ (lane > o)) && (v != v2);
		k = flag ? k : k2;
		v = flag ? v : v2;
	}
}

template <int TPP>
__device__ void ga_block(const KArgs& a, const PopBufs& pb, uint32_t b, const Group<TPP>& G, const GroupSmem& S)
{
	const int P = a.dp.pop_size, NG = a.dp.num_of_genes;
	const uint32_t T = a.ref_threads;
	float* off = S.gen;
	if (b % (uint32_t)P == 0) {
		// elitism: the first warp of the group emulates the reference's T threads
		if (G.rank < 32) {
			const int lane = G.rank;
			const int nw = (int)((T + 31) / 32);
			float wv = FLT_MAX; int wk = -1;   // lane w keeps reference warp w's result
			for (int w = 0; w < nw; w++) {
				const int t = w * 32 + lane;
				float v; int k;
				if (t < P && t < (int)T) { k = (int)b + t; v = pb.e_cur[b + t]; }
				else { k = -1; v = FLT_MAX; }
				if (t < (int)T)
					for (int i = (int)b + (int)T + t; i < (int)b + P; i += (int)T) {
						float e = pb.e_cur[i];
						if (e < v) { k = i; v = e; }
					}
				warp_minimum2(lane, v, k);
				v = __shfl_sync(0xffffffffu, v, 0);
				k = __shfl_sync(0xffffffffu, k, 0);
				if (lane == w) { wv = fminf(kMaxEnergy, v); wk = k; }
			}
			if (lane >= (int)(T / 32)) { wv = FLT_MAX; wk = -1; }
			warp_minimum2(lane, wv, wk);
			if (lane == 0) { S.misc[0] = wk; pb.e[b] = wv; a.evals_new[b] = 0; }
		}
		G.sync();
		const int src = S.misc[0];
		for (int k = G.rank; k < NG; k += TPP) pb.conf[(size_t)b * kGenotypeStride + k] = pb.conf_cur[(size_t)src * kGenotypeStride + k];
		G.sync();
		return;
	}
	float* rn = S.miscf;
	// random numbers [0..3] parents, [4..5] tournaments, [6] crossover, [7..8] points
	for (uint32_t r = G.rank; r < T && r < 10u; r += TPP) {
		uint32_t s = a.prng[b * T + r];
		for (uint32_t i = r; i < 10u; i += T) rn[i] = lcg_float(s);
		a.prng[b * T + r] = s;
	}
	G.sync();
	const int run = (int)b / P;
	int cand[4]; float ce[4];
	for (int i = 0; i < 4; i++) {
		cand[i] = (int)((float)P * rn[i]);
		ce[i] = pb.e_cur[run * P + cand[i]];
	}
	int par[2];
	for (int i = 0; i < 2; i++) {
		if (ce[2 * i] < ce[2 * i + 1]) par[i] = (rn[4 + i] < a.dp.tournament_rate) ? cand[2 * i] : cand[2 * i + 1];
		else par[i] = (rn[4 + i] < a.dp.tournament_rate) ? cand[2 * i + 1] : cand[2 * i];
	}
	const float* p0 = pb.conf_cur + (size_t)(run * P + par[0]) * kGenotypeStride;
	const float* p1 = pb.conf_cur + (size_t)(run * P + par[1]) * kGenotypeStride;
	if (rn[6] < a.dp.crossover_rate) {
		int c0 = (int)((float)(NG - 1) * rn[7]), c1 = (int)((float)(NG - 1) * rn[8]);
		if (c1 < c0) { int t = c1; c1 = c0; c0 = t; }
		for (int g = G.rank; g < NG; g += TPP) {
			if (c0 != c1) off[g] = (g <= c0 || g > c1) ? p0[g] : p1[g];
			else off[g] = (g <= c0) ? p0[g] : p1[g];
		}
	} else {
		for (int g = G.rank; g < NG; g += TPP) off[g] = p0[g];
	}
	G.sync();
	// mutation: reference lane r mutates genes r, r+T, ... with its own stream
	for (uint32_t r = G.rank; r < T; r += TPP) {
		if ((int)r >= NG) continue;
		uint32_t s = a.prng[b * T + r];
		for (int g = (int)r; g < NG; g += (int)T) {
			if (lcg_float(s) < a.dp.mutation_rate) {
				if (g < 3) off[g] += a.dp.abs_max_dmov * (2.0f * lcg_float(s) - 1.0f);
				else { off[g] += a.dp.abs_max_dang * (2.0f * lcg_float(s) - 1.0f); map_angle(off[g]); }
			}
		}
		a.prng[b * T + r] = s;
	}
	G.sync();
	const float e = score_pose<TPP, false>(a.L, off, nullptr, S.pose, G);
	if (G.rank == 0) { pb.e[b] = e; a.evals_new[b] = 1; }
	for (int g = G.rank; g < NG; g += TPP) pb.conf[(size_t)b * kGenotypeStride + g] = off[g];
	G.sync();
}

// The blocks above on the launch's own population buffers.
template <int TPP, int METHOD>
__device__ __forceinline__ void gradient_ls_block(const KArgs& a, uint32_t b, const Group<TPP>& G, const GroupSmem& S)
{ gradient_ls_block<TPP, METHOD>(a, bufs_of(a), b, G, S); }
template <int TPP>
__device__ __forceinline__ void fire_block(const KArgs& a, uint32_t b, const Group<TPP>& G, const GroupSmem& S)
{ fire_block<TPP>(a, bufs_of(a), b, G, S); }
template <int TPP>
__device__ __forceinline__ void sw_block(const KArgs& a, uint32_t b, const Group<TPP>& G, const GroupSmem& S)
{ sw_block<TPP>(a, bufs_of(a), b, G, S); }
template <int TPP>
__device__ __forceinline__ void ga_block(const KArgs& a, uint32_t b, const Group<TPP>& G, const GroupSmem& S)
{ ga_block<TPP>(a, bufs_of(a), b, G, S); }

// Initial population energies (cuda/kernel1.cu:26-55).
template <int TPP>
__device__ void initpop_block(const KArgs& a, const PopBufs& pb, uint32_t b, const Group<TPP>& G, const GroupSmem& S)
{
	const int NG = a.dp.num_of_genes;
	for (int k = G.rank; k < NG; k += TPP) S.gen[k] = pb.conf[(size_t)b * kGenotypeStride + k];
	G.sync();
	const float e = score_pose<TPP, false>(a.L, S.gen, nullptr, S.pose, G);
	if (G.rank == 0) { pb.e[b] = e; a.evals_new[b] = 1; }
	G.sync();
}

template <int TPP>
__device__ __forceinline__ void initpop_block(const KArgs& a, uint32_t b, const Group<TPP>& G, const GroupSmem& S)
{ initpop_block<TPP>(a, bufs_of(a), b, G, S); }

// Stand-alone scorer: energies (and gradients when a.conf_cur != nullptr is
// used as the gradient output) of nblocks genotypes.
template <int TPP, bool GRAD>
__device__ void score_block(const KArgs& a, uint32_t b, const Group<TPP>& G, const GroupSmem& S, float* grads)
{
	const int NG = a.dp.num_of_genes;
	for (int k = G.rank; k < NG; k += TPP) S.gen[k] = a.conf[(size_t)b * kGenotypeStride + k];
	G.sync();
	const float e = score_pose<TPP, GRAD>(a.L, S.gen, S.grad, S.pose, G);
	if (GRAD)
		for (int k = G.rank; k < NG; k += TPP) grads[(size_t)b * kGenotypeStride + k] = S.grad[k];
	if (G.rank == 0) a.e[b] = e;
	G.sync();
}

// The scorer's energy terms (energy only) of nblocks genotypes: a.e[b] the
// energy, out[8b .. 8b+7] the terms (score_pose with TERMS).
template <int TPP>
__device__ void score_terms_block(const KArgs& a, uint32_t b, const Group<TPP>& G, const GroupSmem& S, float* out)
{
	const int NG = a.dp.num_of_genes;
	for (int k = G.rank; k < NG; k += TPP) S.gen[k] = a.conf[(size_t)b * kGenotypeStride + k];
	G.sync();
	const float e = score_pose<TPP, false, false, true>(a.L, S.gen, S.grad, S.pose, G, out + (size_t)b * 8);
	if (G.rank == 0) a.e[b] = e;
	G.sync();
}

}  // namespace adgpu
