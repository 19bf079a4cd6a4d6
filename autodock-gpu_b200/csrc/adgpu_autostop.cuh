// adgpu_autostop.cuh -- AutoStop (host/inc/autostop.hpp:169-222) on the device.
//
// The reference's generation loop copies all R*P current energies to the host
// every as_frequency generations and lets its AutoStop object decide
// (host/src/performdocking.cpp.Cuda:689-698).  Here the resident loop's
// progress kernel takes the same decision on the device, so a docking with
// AutoStop needs no per-check copy and no host round trip.
//
// The statistics are the reference's, operation for operation, with the
// rounding of its host build: float operations where its operands are float,
// double where a double literal promotes them, no fused multiply-adds
// (explicitly rounded intrinsics).  Which energies fall below the threshold,
// and into which bin, is found by the whole block in parallel; the float sums
// that depend on order are then taken by one thread in the reference's order
// (runs, then entities).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace adgpu {

struct AutoStopState {
	int first_time, autostopped;
	float threshold, threshold_used, thres_stddev, curr_avg, curr_std;
	unsigned int roll_count, bestN;
	float rolling[16];
	float delta_energy, overall_best_energy;
	int num_runs;
	unsigned int pop_size, Ntop, Ncream;
	float stopstd;
	unsigned int as_frequency;
};

// The AutoStop constructor (autostop.hpp:131-163), host side.
inline void autostop_init(AutoStopState& s, int pop_size, int num_runs, float stopstd, unsigned int as_frequency)
{
	s = AutoStopState();
	s.num_runs = num_runs;
	s.pop_size = (unsigned int)pop_size;
	s.Ntop = (unsigned int)pop_size;
	s.Ncream = (unsigned int)pop_size / 10;
	s.stopstd = stopstd;
	s.as_frequency = as_frequency;
	s.first_time = 1;
	s.autostopped = 0;
	s.threshold = 1 << 24;
	s.threshold_used = s.threshold;
	s.thres_stddev = s.threshold;
	s.curr_avg = -(1 << 24);
	s.curr_std = s.thres_stddev;
	s.roll_count = 0;
	s.bestN = 1;
	s.delta_energy = (float)(2.0 * (double)s.thres_stddev / (double)s.Ntop);
	s.overall_best_energy = 1 << 24;
}

// Floats of the statistics array average_sd2_N: (pop_size + 1) * 3.
inline size_t autostop_stats_floats(int pop_size) { return (size_t)(pop_size + 1) * 3; }

__device__ __forceinline__ float as_average(const float* a)
{
	if (a[2] < 1.0f) return 0.0f;
	return __fdiv_rn(a[0], a[2]);
}

__device__ __forceinline__ float as_stddev(const float* a)
{
	if (a[2] < 1.0f) return 0.0f;
	const float sq = __fsub_rn(__fmul_rn(a[1], a[2]), __fmul_rn(a[0], a[0]));
	if (((double)fabsf(sq) <= 0.000001) || (sq < 0.0f)) return 0.0f;
	return __fdiv_rn(__fsqrt_rn(sq), a[2]);
}

// tabulate_energies (autostop.hpp:83-104) with the whole block: thread t scans
// a contiguous chunk, the chunks' below-threshold entries are compacted in
// order into buf_e/buf_m (bin Ntop = none), and thread 0 sums them in order.
__device__ void as_tabulate(AutoStopState& s, float* a, float* buf_e, uint16_t* buf_m, const float* energies, int n,
                            int* s_count, float* s_best)
{
	const int T = blockDim.x, t = threadIdx.x;
	const int chunk = (n + T - 1) / T, i0 = t * chunk, i1 = min(n, i0 + chunk);
	const double base = __dsub_rn((double)s.threshold, __dmul_rn(2.0, (double)s.thres_stddev));
	int cnt = 0;
	float best = 1 << 24;
	for (int i = i0; i < i1; i++) {
		const float e = energies[i];
		if (e < best) best = e;
		cnt += e < s.threshold;
	}
	s_count[t] = cnt;
	s_best[t] = best;
	__syncthreads();
	if (t == 0) {
		int run = 0;
		float b = 1 << 24;
		for (int k = 0; k < T; k++) { const int c = s_count[k]; s_count[k] = run; run += c; if (s_best[k] < b) b = s_best[k]; }
		s_count[T] = run;
		s.overall_best_energy = b;
	}
	__syncthreads();
	int pos = s_count[t];
	for (int i = i0; i < i1; i++) {
		const float e = energies[i];
		if (!(e < s.threshold)) continue;
		unsigned int m = 0;
		for (; m < s.Ntop; m++)
			if ((double)e < __dadd_rn(base, (double)__fmul_rn((float)m, s.delta_energy))) break;
		buf_e[pos] = e;
		buf_m[pos] = (uint16_t)m;
		pos++;
	}
	__syncthreads();
	if (t == 0) {
		const int total = s_count[T];
		for (int k = 0; k < total; k++) {
			const float e = buf_e[k];
			a[0] = __fadd_rn(a[0], e);
			a[1] = __fadd_rn(a[1], __fmul_rn(e, e));
			a[2] = (float)__dadd_rn((double)a[2], 1.0);
			const unsigned int m = buf_m[k];
			if (m < s.Ntop) {
				float* b = a + 3 * (m + 1);
				b[0] = __fadd_rn(b[0], e);
				b[1] = __fadd_rn(b[1], __fmul_rn(e, e));
				b[2] = (float)__dadd_rn((double)b[2], 1.0);
			}
		}
	}
	__syncthreads();
}

// set_stats (autostop.hpp:106-129), one thread.
__device__ void as_set_stats(AutoStopState& s, float* a)
{
	s.curr_avg = as_average(a);
	s.curr_std = as_stddev(a);
	s.bestN = (unsigned int)a[2];
	a[0] = 0.0f; a[1] = 0.0f; a[2] = 0.0f;
	unsigned int lowest_energy = 0;
	for (unsigned int m = 0; m < s.Ntop; m++) {
		float* b = a + 3 * (m + 1);
		if ((b[2] >= 1.0f) && (lowest_energy < s.Ncream)) {
			if ((a[2] < 4.0f) ||
			    (double)fabsf(__fsub_rn(as_average(a), as_average(b))) < __dmul_rn(2.0, (double)s.stopstd)) {
				a[0] = __fadd_rn(a[0], b[0]);
				a[1] = __fadd_rn(a[1], b[1]);
				a[2] = __fadd_rn(a[2], b[2]);
				lowest_energy++;
			}
		}
	}
	if (lowest_energy > 0) {
		s.curr_avg = as_average(a);
		s.curr_std = as_stddev(a);
		s.bestN = (unsigned int)a[2];
	}
}

// check_if_satisfactory (autostop.hpp:169-222) with the whole block; the
// result is s.autostopped.  scratch: s_count[blockDim.x + 1], s_best[blockDim.x].
__device__ void autostop_check(AutoStopState& s, float* a, float* buf_e, uint16_t* buf_m, const float* energies,
                               int generation_cnt, int* s_count, float* s_best)
{
	const int n = s.num_runs * (int)s.pop_size;
	const int nstats = (int)(s.pop_size + 1) * 3;
	const int reps = 1 + 8 * (generation_cnt == 0);
	for (int count = 0; count < reps; count++) {
		__syncthreads();
		if (!((double)fabsf(s.curr_avg) > 0.00001)) break;    // uniform: every thread reads the same state
		__syncthreads();
		if (threadIdx.x == 0) s.threshold_used = s.threshold;
		for (int k = threadIdx.x; k < nstats; k += blockDim.x) a[k] = 0.0f;
		__syncthreads();
		as_tabulate(s, a, buf_e, buf_m, energies, n, s_count, s_best);
		if (threadIdx.x == 0) {
			if (s.first_time) {
				s.curr_avg = as_average(a);
				s.curr_std = as_stddev(a);
				s.bestN = (unsigned int)a[2];
				s.thres_stddev = s.curr_std;
				s.threshold = __fadd_rn(s.curr_avg, s.thres_stddev);
				s.delta_energy = (float)__ddiv_rn(__dmul_rn(2.0, (double)s.thres_stddev), (double)(s.Ntop - 1));
				s.first_time = 0;
			} else {
				as_set_stats(s, a);
				if (s.curr_std < __fmul_rn(0.5f, s.stopstd)) s.thres_stddev = s.stopstd;
				else s.thres_stddev = s.curr_std;
				s.threshold = __fadd_rn(s.curr_avg, __fdiv_rn(__fmul_rn((float)s.Ncream, s.thres_stddev), (float)s.bestN));
				s.delta_energy = (float)__ddiv_rn(__dmul_rn(2.0, (double)s.thres_stddev), (double)(s.Ntop - 1));
			}
		}
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		float* r = s.rolling;
		const unsigned int rc = s.roll_count;
		const float bn = (float)s.bestN;
		r[4 * rc] = __fmul_rn(s.curr_avg, bn);
		r[4 * rc + 1] = __fmul_rn(__fadd_rn(__fmul_rn(s.curr_std, s.curr_std), __fmul_rn(s.curr_avg, s.curr_avg)), bn);
		r[4 * rc + 2] = bn;
		r[4 * rc + 3] = s.overall_best_energy;
		s.roll_count = (rc + 1) % 4;
		a[0] = __fadd_rn(__fadd_rn(__fadd_rn(r[0], r[4]), r[8]), r[12]);
		a[1] = __fadd_rn(__fadd_rn(__fadd_rn(r[1], r[5]), r[9]), r[13]);
		a[2] = __fadd_rn(__fadd_rn(__fadd_rn(r[2], r[6]), r[10]), r[14]);
		float best_avg = __fadd_rn(__fadd_rn(__fadd_rn(r[3], r[7]), r[11]), r[15]);
		best_avg = __fdiv_rn(best_avg, 4.0f);
		float best_var = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(r[3], r[3]), __fmul_rn(r[7], r[7])), __fmul_rn(r[11], r[11])),
		                           __fmul_rn(r[15], r[15]));
		best_var = __fdiv_rn(best_var, 4.0f);
		best_var = __fsub_rn(best_var, __fmul_rn(best_avg, best_avg));
		if ((as_stddev(a) < s.stopstd) && (generation_cnt >= (int)(4 * s.as_frequency)) && (best_var <= 0.00002f))
			s.autostopped = 1;
	}
	__syncthreads();
}

}  // namespace adgpu
