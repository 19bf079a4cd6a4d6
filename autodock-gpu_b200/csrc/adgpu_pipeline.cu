// adgpu_pipeline.cu -- the plain docking loop (docking_with_gpu's generation
// loop, host/src/performdocking.cpp.Cuda:684-831) as one persistent kernel in
// which the runs of the ligand advance independently.
//
// The reference runs a generation as three grid-wide kernels (GA, local
// search, eval sums) and tests progress between generations on the mean
// evaluations over all runs (check_progress, :908-942).  Local searches stop
// on their own step-size test, so each local-search launch ends with its
// longest searches running alone: with the cfg2 ligand (100 runs x 150
// ADADELTA searches, mean 67 and up to 300 iterations) a third of the
// launch's pose-group time is idle.
//
// Here every run's generation is split into one task per entity -- the GA
// step that makes the entity (elitism, or tournaments, crossover, mutation
// and scoring) followed by its local search, both on the entity's own PRNG
// states in the reference's order -- and a run starts its next generation as
// soon as its own last task ends.  Each run hands out the entities of its
// current generation from one counter (generation << 32 | entities taken);
// a pose group scans the runs' counters and takes an entity of a run in the
// oldest open generation, so the runs that gate the next stop test are never
// queued behind runs that are ahead of them.  The stop
// test keeps the reference's semantics exactly: check g (before generation g)
// uses the evaluations of all runs after generation g-1, so it is taken by
// whichever pose group completes the last run's generation g-1.  Runs may
// run ahead of that decision by up to nbuf-1 generations (nbuf population
// buffers, 4 or 8): generation g reads buffer g % nbuf and writes buffer
// (g+1) % nbuf, which holds the result of generation g - nbuf; that result is
// needed only if check g - nbuf + 1 says stop, so generation g may start once
// that check has said continue.  Generations the evaluation count will not
// reach are not started: each check projects the generation at which the
// stop will come from the evaluations the last generation added, and runs
// wait at one generation past it until the next check.  When a check says stop, the generations
// already run past it are discarded: their evaluations are taken back off the
// per-run counters and the final population is the one the reference ends
// with.  Every run performs exactly the reference's operations on its own
// population and PRNG states (local-search entity l of run r uses the states
// of GA block r*P + l, inside its own run, because the local-search rate is
// 100 %), so populations, energies and evaluation counts are bit-identical
// to the generation-synchronous loop; only the PRNG states and the per-entity
// evaluation counters of the discarded generations differ.
#include <cuda_runtime.h>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "adgpu_kernels.cuh"
#include "adgpu_queue.cuh"
#include "adgpu_pipeline.h"

// CTAs per SM the persistent kernel is compiled for.  Gradient local
// searches: 5 CTAs of 4 pose groups; with 6 the SM's throughput is the same
// (the scorer is issue bound), but the cfg2 ADADELTA docking's 100 runs x
// 150 entities then leave runs waiting for the stop test (pose groups 95 %
// busy against 99 %, 158 against 165 M evaluations/s on B200).  Solis-Wets
// scores energies only, in fewer registers, and gains from the extra warps.
#ifndef ADGPU_PIPE_MIN_CTAS
#define ADGPU_PIPE_MIN_CTAS 5
#endif
#ifndef ADGPU_PIPE_MIN_CTAS_SW
#define ADGPU_PIPE_MIN_CTAS_SW 7
#endif

namespace adgpu {

constexpr int kPipeThreads = 128;
constexpr uint32_t kPipeRunShift = 11;         // a taken task: run << 11 | entity
constexpr int kRetired = 0x40000000;           // started[r] of a retired run


struct PipeCtl {
	QueueCtl q;                               // q.alive = runs not retired, q.err, accounting
	int done;                                 // every run has retired
	int dec;                                  // checks 0 .. dec-1 have said continue
	int stop_gen;                             // -1, or the generations run (the check that said stop)
	unsigned long long parks;                 // times a run waited for a check before its next generation
	unsigned long long executed;              // evaluations executed, discarded generations included
	unsigned long long last_tot;              // evaluations over all runs at the last check
	int limit;                                // generations above this one do not start (projected stop)
	int pad;
	unsigned long long acc[kPipeBufs];        // per generation slot: sum over runs of the evaluations after it
	int fin[kPipeBufs];                       // per generation slot: runs that completed it
};

struct PipeArgs {
	KArgs ka;                   // tables, dockpars, PRNG states, evaluation counters
	PopBufs bufs[kPipeBufs];    // generation slot k: conf_cur/e_cur = buffer k, conf/e = buffer (k+1) % nbuf
	unsigned long long* next;   // R: the run's open generation << 32 | its entities taken
	long long idle_ns;          // a pose group that finds no task for this long gives up (error)
	PipeCtl* ctl;
	int* started;               // R: generations started (claimed), kRetired once retired
	int* done;                  // R: generations completed (or abandoned after a stop)
	int* comp;                  // R: generations whose evaluations are in evals_runs
	int* pending;               // R: tasks of the run's current phase not yet finished
	int* inc;                   // R * kPipeBufs: evaluations each generation slot added
	int runs, pop;
	int nbuf;                   // population buffers in use (4 or 8): look-ahead nbuf-1 generations
	unsigned long long max_evals;
	unsigned int max_gens;
	int group_bytes;            // shared memory per pose group (header + scratch)
};

struct PipeHdr {
	unsigned long long pos;
	long long t_enter, t_task;       // worker accounting (rank 0; globaltimer ns)
	unsigned long long busy, ntask, nevals;
	int task, gen, last, decider, stopped, isum;
};
constexpr int kPipeHdrBytes = (int)((sizeof(PipeHdr) + 15) / 16 * 16);

__device__ __forceinline__ int vload(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

// Starts run r's next generation when the checks allow it, or retires the run
// once a check has said stop.  Called by the run's own pose group after each
// generation and by the group that publishes a check (for runs parked ahead
// of it); the CAS on started[r] lets exactly one caller act.
__device__ void pipe_try_start(const PipeArgs& p, int r)
{
	const int d = vload(p.done + r);
	if (vload(p.started + r) != d) return;            // running, or retired
	volatile PipeCtl* vc = p.ctl;
	if (vc->stop_gen >= 0) {
		// the last run to retire ends every worker
		if (atomicCAS(p.started + r, d, kRetired) == d && atomicSub(&p.ctl->q.alive, 1) == 1) {
			__threadfence();
			vc->done = 1;
		}
		return;
	}
	if (d - p.nbuf + 1 >= vc->dec || d > vc->limit) { // parked: check d-nbuf+1 still open, or past the projected stop
		atomicAdd(&p.ctl->parks, 1ull);
		return;
	}
	if (atomicCAS(p.started + r, d, d + 1) != d) return;
	p.pending[r] = p.pop;
	__threadfence();
	// open generation d's entities
	atomicExch(p.next + r, (unsigned long long)d << 32);
}

// An entity to work on: the first warp of the pose group scans the runs'
// counters for the lowest open generation with entities left (ties: the
// first run at or after this group's own offset, so that groups spread over
// the runs), and takes one with an atomicAdd; a take past the run's last
// entity only sends the scan round again.  Returns run << 11 | entity and the
// generation in *gen, or -1 once every run has retired (or after idle_ns with
// nothing to take: an error).
template <int TPP>
__device__ int pipe_take(const PipeArgs& p, int worker, const Group<TPP>& G, int* gen)
{
	volatile PipeCtl* vc = p.ctl;
	const int lane = G.rank;            // called by the group's first warp only
	const int R = p.runs, P = p.pop;
	const int off = worker % R;
	long long idle_since = -1;
	int backoff = 64;
	for (int spins = 0; spins < (1 << 30); spins++) {
		if (vc->done) return -1;
		unsigned long long best = ~0ull;
		for (int r = lane; r < R; r += 32) {
			const unsigned long long v = *reinterpret_cast<const volatile unsigned long long*>(p.next + r);
			if ((uint32_t)v < (uint32_t)P) {
				const unsigned long long key = ((v >> 32) << 32) | (uint32_t)((r - off + R) % R);
				best = key < best ? key : best;
			}
		}
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) {
			const unsigned long long x = __shfl_xor_sync(0xffffffffu, best, o);
			best = x < best ? x : best;
		}
		if (best != ~0ull) {
			const int r = (int)(((uint32_t)best + off) % (uint32_t)R);
			unsigned long long old = 0;
			if (lane == 0) old = atomicAdd(p.next + r, 1ull);
			old = __shfl_sync(0xffffffffu, old, 0);
			if ((uint32_t)old < (uint32_t)P) {
				__threadfence();
				*gen = (int)(old >> 32);
				return (r << kPipeRunShift) | (int)(uint32_t)old;
			}
			continue;
		}
		const long long now = global_ns();
		if (idle_since < 0) idle_since = now;
		else if (now - idle_since > p.idle_ns) break;
		__nanosleep(backoff);
		if (backoff < 4096) backoff *= 2;
	}
	if (lane == 0) atomicExch(&p.ctl->q.err, 2);
	return -1;
}

template <int TPP, int LSMET>
__device__ void pipe_worker(const PipeArgs& p)
{
	extern __shared__ __align__(16) char smem[];
	const int local = threadIdx.x / TPP;
	char* base = smem + (size_t)local * p.group_bytes;
	PipeHdr& H = *reinterpret_cast<PipeHdr*>(base);
	const LigDev& L0 = p.ka.L;
	const GroupSmem S = carve_group(base + kPipeHdrBytes, L0.natoms, L0.ntors, 64, TPP);
	Group<TPP> G;
	G.rank = threadIdx.x % TPP;
	G.bar_id = 1 + local;
	G.red = S.red;
	const int P = p.pop, R = p.runs;
	if (G.rank == 0) { H.t_enter = global_ns(); H.t_task = 0; H.busy = 0; H.ntask = 0; H.nevals = 0; }
	const int worker = blockIdx.x * (kPipeThreads / TPP) + local;
	for (;;) {
		if (G.rank < 32) {
			if (G.rank == 0 && H.t_task) H.busy += (unsigned long long)(global_ns() - H.t_task);
			int gen = 0;
			const int task = pipe_take<TPP>(p, worker, G, &gen);
			if (G.rank == 0) {
				H.task = task;
				H.t_task = task >= 0 ? global_ns() : 0;
				H.ntask += task >= 0;
				H.gen = gen;
				H.stopped = reinterpret_cast<volatile PipeCtl*>(p.ctl)->stop_gen >= 0;
			}
		}
		G.sync();
		const int task = H.task;
		if (task < 0) break;
		const int run = task >> kPipeRunShift;
		const int ent = task & ((1 << kPipeRunShift) - 1);
		const int g = H.gen;
		// a generation past a check that said stop is discarded: its tasks
		// only count down
		if (!H.stopped) {
			const KArgs& a = p.ka;
			const PopBufs pb = p.bufs[g & (p.nbuf - 1)];
			const uint32_t b = (uint32_t)(run * P + ent);
			ga_block<TPP>(a, pb, b, G, S);
			// num_of_lsentities == pop_size: local-search block b is entity b
			if constexpr (LSMET == LS_SW) sw_block<TPP>(a, pb, b, G, S);
			else if constexpr (LSMET == LS_AD) gradient_ls_block<TPP, LS_AD>(a, pb, b, G, S);
			else if constexpr (LSMET == LS_ADAM) gradient_ls_block<TPP, LS_ADAM>(a, pb, b, G, S);
			else fire_block<TPP>(a, pb, b, G, S);
		}
		__threadfence();
		G.sync();
		if (G.rank == 0) {
			if (!H.stopped) H.nevals += (unsigned long long)p.ka.evals_new[run * P + ent];
			H.last = (atomicSub(p.pending + run, 1) == 1);
		}
		G.sync();
		if (!H.last) continue;
		__threadfence();
		// ---- generation g of this run is complete (or abandoned after a stop) ----
		int s = 0;
		if (!H.stopped)
			for (int i = G.rank; i < P; i += TPP) s += p.ka.evals_new[run * P + i];
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
		if constexpr (TPP > 32) {
			if (G.rank == 0) H.isum = 0;
			G.sync();
			if ((G.rank & 31) == 0) atomicAdd(&H.isum, s);
			G.sync();
			s = H.isum;
		}
		if (G.rank == 0) {
			H.decider = 0;
			const int slot = g & (p.nbuf - 1);
			if (!H.stopped) {
				// the eval sum of the run (cuda/kernel2.cu:26-52)
				int* er = p.ka.evals_runs + run;
				const int cum = *er + s;
				*er = cum;
				p.inc[run * kPipeBufs + slot] = s;
				p.comp[run] = g + 1;
				__threadfence();
				atomicAdd(&p.ctl->acc[slot], (unsigned long long)cum);
				__threadfence();
				if (atomicAdd(&p.ctl->fin[slot], 1) + 1 == R) {
					// every run has completed generation g: check g+1
					// (check_progress, performdocking.cpp.Cuda:908-942)
					const unsigned long long tot = atomicExch(&p.ctl->acc[slot], 0ull);
					atomicExch(&p.ctl->fin[slot], 0);
					const double ev = (double)tot / (double)R / (double)p.max_evals * 100.0;
					const double gp = (double)(g + 1) / (double)p.max_gens * 100.0;
					__threadfence();
					volatile PipeCtl* vc = p.ctl;
					// a generation run past a stop can still complete everywhere
					// (its last tasks were taken before the stop was seen)
					if (vc->stop_gen < 0) {
						if ((ev > gp ? ev : gp) >= 100.0) {
							vc->stop_gen = g + 1;
						} else {
							// project the stop: generations g+1 .. g+k still to run
							// at the rate generation g added; start none past g+k+1
							const unsigned long long target = (unsigned long long)R * p.max_evals;
							const unsigned long long delta = tot > p.ctl->last_tot ? tot - p.ctl->last_tot : 1ull;
							const unsigned long long k = (target - tot + delta - 1) / delta;
							long long lim = (long long)g + (long long)k + 1;
							if (lim > (long long)p.max_gens - 1) lim = (long long)p.max_gens - 1;
							if (lim > 0x3fffffff) lim = 0x3fffffff;
							vc->limit = (int)lim;
							p.ctl->last_tot = tot;
							vc->dec = g + 2;
						}
					}
					H.decider = 1;
				}
			}
			*reinterpret_cast<volatile int*>(p.done + run) = g + 1;
			__threadfence();
		}
		G.sync();
		if (H.decider) {
			__threadfence();
			for (int r = G.rank; r < R; r += TPP) pipe_try_start(p, r);
			G.sync();
		}
		if (G.rank == 0) pipe_try_start(p, run);
		G.sync();
	}
	if (G.rank == 0) {
		atomicAdd(&p.ctl->q.busy_ns, H.busy);
		atomicAdd(&p.ctl->executed, H.nevals);
		atomicAdd(&p.ctl->q.tasks, H.ntask);
		atomicAdd(&p.ctl->q.workers, 1);
		atomicMin(&p.ctl->q.t_first, (unsigned long long)H.t_enter);
		atomicMax(&p.ctl->q.t_last, (unsigned long long)global_ns());
	}
}

constexpr int pipe_min_ctas(int lsmet) { return lsmet == LS_SW ? ADGPU_PIPE_MIN_CTAS_SW : ADGPU_PIPE_MIN_CTAS; }

template <int TPP, int LSMET>
__global__ void __launch_bounds__(kPipeThreads, pipe_min_ctas(LSMET)) pipe_kernel(const PipeArgs p)
{
	pipe_worker<TPP, LSMET>(p);
}

// Check 0 (before the first generation) and the first generation's GA tasks.
__global__ void __launch_bounds__(256) pipe_init_kernel(PipeArgs p)
{
	__shared__ unsigned long long tot;
	if (threadIdx.x == 0) tot = 0;
	__syncthreads();
	unsigned long long s = 0;
	for (int r = threadIdx.x; r < p.runs; r += blockDim.x) s += (unsigned long long)p.ka.evals_runs[r];
	atomicAdd(&tot, s);
	__syncthreads();
	const double ev = (double)tot / (double)p.runs / (double)p.max_evals * 100.0;
	const bool stop = ev >= 100.0;     // generations 0 of max_gens >= 1
	for (int r = threadIdx.x; r < p.runs; r += blockDim.x) {
		p.started[r] = stop ? kRetired : 1;
		p.done[r] = 0;
		p.comp[r] = 0;
		p.pending[r] = p.pop;
		p.next[r] = stop ? (unsigned long long)(uint32_t)p.pop : 0ull;   // generation 0 open, or nothing to take
	}
	if (threadIdx.x == 0) {
		PipeCtl* c = p.ctl;
		c->q.alive = stop ? 0 : p.runs;
		c->done = stop ? 1 : 0;
		c->dec = 1;
		c->stop_gen = stop ? 0 : -1;
		c->q.t_first = ~0ull;
		c->last_tot = tot;
		c->limit = (int)(p.max_gens - 1 < 0x3fffffffu ? p.max_gens - 1 : 0x3fffffffu);
	}
}

// Takes the evaluations of discarded generations back off the per-run
// counters.  out: generations run, runs not retired, task error, most
// generations a run ran past the stop, then the accounting (busy ns, tasks,
// first start, last exit, parks, pose groups).
__global__ void __launch_bounds__(256) pipe_final_kernel(PipeArgs p, long long* out)
{
	__shared__ int past;
	if (threadIdx.x == 0) past = 0;
	__syncthreads();
	const int G = p.ctl->stop_gen;
	for (int r = threadIdx.x; r < p.runs; r += blockDim.x)
		if (G >= 0) {
			for (int k = G; k < p.comp[r]; k++) p.ka.evals_runs[r] -= p.inc[r * kPipeBufs + (k & (p.nbuf - 1))];
			atomicMax(&past, p.done[r] - G);
		}
	__syncthreads();
	if (threadIdx.x == 0) {
		const QueueCtl& q = p.ctl->q;
		out[0] = G; out[1] = q.alive; out[2] = q.err; out[3] = past;
		out[4] = (long long)q.busy_ns; out[5] = (long long)q.tasks;
		out[6] = q.workers ? (long long)(q.t_last - q.t_first) : 0;
		out[7] = (long long)p.ctl->parks; out[8] = q.workers; out[9] = (long long)p.ctl->executed;
	}
}

// Initial check and tasks, the persistent launch, the final accounting; the
// grid is sized from the kernel's occupancy (persistent: every pose group a
// worker) and capped by the entities a generation offers.
template <int TPP, int LSMET>
static adgpu_status launch_pipe(PipeArgs p, long long* d_out, cudaStream_t st)
{
	auto kfn = pipe_kernel<TPP, LSMET>;
	const int gpc = kPipeThreads / TPP;
	const int bytes = p.group_bytes * gpc;
	if (bytes > 48 * 1024) ADGPU_CUDA_RET(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes), "pipeline smem");
	const int pct = smem_carveout_pct(bytes, pipe_min_ctas(LSMET));
	if (pct >= 0) ADGPU_CUDA_RET(cudaFuncSetAttribute(kfn, cudaFuncAttributePreferredSharedMemoryCarveout, pct), "pipeline carveout");
	int per_sm = 0, dev = 0, sms = 0;
	ADGPU_CUDA_RET(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kPipeThreads, bytes), "pipeline occupancy");
	if (per_sm < 1) return fail(ADGPU_ERR_LIMIT, "pipeline kernel does not fit on an SM");
	ADGPU_CUDA_RET(cudaGetDevice(&dev), "device");
	ADGPU_CUDA_RET(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "sm count");
	const long useful = ((long)p.runs * p.pop + gpc - 1) / gpc;
	long grid = (long)per_sm * sms;
	if (grid > useful) grid = useful;
	pipe_init_kernel<<<1, 256, 0, st>>>(p);
	ADGPU_CUDA_RET(cudaGetLastError(), "pipeline init");
	kfn<<<(int)grid, kPipeThreads, bytes, st>>>(p);
	ADGPU_CUDA_RET(cudaGetLastError(), "pipeline launch");
	pipe_final_kernel<<<1, 256, 0, st>>>(p, d_out);
	ADGPU_CUDA_RET(cudaGetLastError(), "pipeline final");
	return ADGPU_OK;
}

bool pipeline_applies(const adgpu_dockpars& dp, uint32_t runs)
{
	return dp.num_of_lsentities == (uint32_t)dp.pop_size && dp.lsearch_rate != 0.0f && dp.pop_size > 0 &&
	       dp.pop_size <= (1 << kPipeRunShift) && runs > 0 && runs < (1u << (31 - kPipeRunShift));
}

// Threads per pose of the pipelined loop: the smallest group that still has
// about four entities per pose group in a generation (runs * pop_size tasks
// over SMs x 6 CTAs x 128/TPP groups).  Runs advance independently and a
// generation's entities are handed out oldest generation first, so a launch
// no longer ends each generation with its longest searches running alone,
// and one warp per pose gives the most evaluations per SM when there is work
// for all of them (B200, cfg2, 100 runs: ADADELTA 158 vs 148, Solis-Wets 255
// vs 249, ADAM 174 vs 155, FIRE 140 vs 119 M evals/s against 64).  With few
// runs a run's chain of generations decides, and larger groups shorten it
// (16 uneven ligands of 20 runs, ADADELTA: 54, 86 and 102 M evals/s at 32,
// 64 and 128).
int pipeline_default_tpp(int lsmet, long tasks)
{
	(void)lsmet;
	int dev = 0, sms = 148;
	if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	for (int tpp = 32; tpp < 128; tpp *= 2)
		if (tasks >= 4L * sms * ADGPU_PIPE_MIN_CTAS * (kPipeThreads / tpp)) return tpp;
	return 128;
}

// Population buffers (look-ahead + 1): with 32 threads per pose a run's
// generation takes longer (its longest search runs on one warp), so runs are
// let further ahead of the slowest (ADADELTA: pose groups 94 % busy with 8
// buffers, 94 % with 4; with 64 threads 99 % either way).
int pipeline_buffers(int tpp)
{
	if (const char* e = getenv("ADGPU_PIPELINE_BUFFERS")) {
		const int v = atoi(e);
		if (v == 4 || v == 8) return v;
	}
	return tpp == 32 ? 8 : 4;
}

adgpu_status dock_pipelined(const KArgs& base, PipeScratch& sc, int lsmet, int tpp, uint32_t runs,
                            uint64_t max_evals, uint32_t max_gens, float* c1, float* e1, float* c2, float* e2,
                            int* final_is_second, uint32_t* generations)
{
	const adgpu_dockpars& dp = base.dp;
	if (!pipeline_applies(dp, runs)) return fail(ADGPU_ERR_ARG, "pipelined docking needs a 100 % local-search rate");
	if (tpp == 0) tpp = pipeline_default_tpp(lsmet, (long)runs * dp.pop_size);
	if (tpp != 32 && tpp != 64 && tpp != 128) return fail(ADGPU_ERR_ARG, "threads per pose must be 32, 64 or 128");
	const int P = dp.pop_size;
	const size_t n = (size_t)runs * P;
	const int nbuf = pipeline_buffers(tpp);
	// scratch: nbuf-2 more population buffers, per-run counters, control
	auto al = [](size_t b) { return (b + 255) / 256 * 256; };
	const size_t conf1 = al(n * kGenotypeStride * 4), e1b = al(n * 4);
	const size_t o_conf = 0, conf_b = conf1 * (nbuf - 2);
	const size_t o_e = o_conf + conf_b, e_b = e1b * (nbuf - 2);
	const size_t o_slots = o_e + e_b, slots_b = al((size_t)runs * 8);
	const size_t o_runs = o_slots + slots_b, runs_b = al((size_t)runs * 4) * 4 + al((size_t)runs * kPipeBufs * 4);
	const size_t o_ctl = o_runs + runs_b, ctl_b = al(sizeof(PipeCtl)) + 256;
	const size_t total = o_ctl + ctl_b;
	if (sc.bytes < total) {
		if (sc.mem) cudaFree(sc.mem);
		sc.mem = nullptr; sc.bytes = 0;
		ADGPU_CUDA_RET(cudaMalloc(&sc.mem, total), "pipeline scratch");
		sc.bytes = total;
	}
	if (!sc.host_out) ADGPU_CUDA_RET(cudaMallocHost(&sc.host_out, 16 * sizeof(long long)), "pipeline readback");
	char* m = static_cast<char*>(sc.mem);
	float* conf[kPipeBufs] = {c1, c2};
	float* en[kPipeBufs] = {e1, e2};
	for (int k = 2; k < nbuf; k++) {
		conf[k] = reinterpret_cast<float*>(m + o_conf + conf1 * (k - 2));
		en[k] = reinterpret_cast<float*>(m + o_e + e1b * (k - 2));
	}
	PipeArgs p;
	memset(&p, 0, sizeof(p));
	p.ka = base;
	p.ka.ref_threads = 64;
	p.ka.stop_flag = nullptr;
	p.ka.work_counter = nullptr;
	p.ka.nblocks = 0;
	p.ka.conf_cur = p.ka.e_cur = nullptr;
	p.ka.conf = p.ka.e = nullptr;
	p.nbuf = nbuf;
	for (int k = 0; k < nbuf; k++)
		p.bufs[k] = PopBufs{conf[k], en[k], conf[(k + 1) % nbuf], en[(k + 1) % nbuf]};
	p.next = reinterpret_cast<unsigned long long*>(m + o_slots);
	p.idle_ns = 2000000000ll;
	int* ri = reinterpret_cast<int*>(m + o_runs);
	const size_t rs = al((size_t)runs * 4) / 4;
	p.started = ri; p.done = ri + rs; p.comp = ri + 2 * rs; p.pending = ri + 3 * rs; p.inc = ri + 4 * rs;
	p.ctl = reinterpret_cast<PipeCtl*>(m + o_ctl);
	long long* d_out = reinterpret_cast<long long*>(m + o_ctl + al(sizeof(PipeCtl)));
	p.runs = (int)runs; p.pop = P;
	p.max_evals = max_evals; p.max_gens = max_gens;
	p.group_bytes = kPipeHdrBytes + group_smem_bytes(base.L.natoms, base.L.ntors, 64, tpp);

	cudaStream_t st = 0;   // the legacy stream: ordered after the caller's initial-population calls
	// the library's population buffers start as zeros, like the caller's
	// second buffer: genes past num_of_genes are never written
	ADGPU_CUDA_RET(cudaMemsetAsync(m + o_conf, 0, conf_b + e_b, st), "pipeline buffers");
	ADGPU_CUDA_RET(cudaMemsetAsync(p.ctl, 0, sizeof(PipeCtl), st), "pipeline control");
	adgpu_status rc = ADGPU_OK;
#define ADGPU_PIPE_LSMET(T) \
	switch (lsmet) { \
	case 0: rc = launch_pipe<T, LS_SW>(p, d_out, st); break; \
	case 1: rc = launch_pipe<T, LS_AD>(p, d_out, st); break; \
	case 2: rc = launch_pipe<T, LS_ADAM>(p, d_out, st); break; \
	default: rc = launch_pipe<T, LS_FIRE>(p, d_out, st); break; \
	}
	switch (tpp) {
	case 32: ADGPU_PIPE_LSMET(32) break;
	case 64: ADGPU_PIPE_LSMET(64) break;
	default: ADGPU_PIPE_LSMET(128) break;
	}
#undef ADGPU_PIPE_LSMET
	if (rc != ADGPU_OK) return rc;
	ADGPU_CUDA_RET(cudaMemcpyAsync(sc.host_out, d_out, 10 * sizeof(long long), cudaMemcpyDeviceToHost, st), "pipeline readback");
	ADGPU_CUDA_RET(cudaStreamSynchronize(st), "pipeline docking");
	const long long* o = sc.host_out;
	const int G = (int)o[0], alive = (int)o[1], err = (int)o[2];
	adgpu_dock_stats& ds = sc.stats;
	memset(&ds, 0, sizeof(ds));
	ds.pipelined = 1;
	ds.threads_per_pose = tpp;
	ds.pose_groups = (int)o[8];
	ds.generations = G < 0 ? 0 : (uint32_t)G;
	ds.generations_discarded = (uint32_t)(o[3] > 0 ? o[3] : 0);
	ds.busy_s = 1e-9 * (double)o[4];
	ds.tasks = (uint64_t)o[5];
	ds.span_s = 1e-9 * (double)o[6];
	ds.parks = (uint64_t)o[7];
	ds.evals_executed = (uint64_t)o[9];
	ds.buffers = nbuf;
	if (err != 0 || alive != 0 || G < 0)
		return fail(ADGPU_ERR_TIMEOUT, "pipelined docking: a bounded device wait gave up (task error " + std::to_string(err) +
		                                ", runs still active " + std::to_string(alive) + ")");
	*generations = (uint32_t)G;
	*final_is_second = G & 1;
	const int fb = G & (nbuf - 1);
	if (fb >= 2) {
		// the final population sits in a library buffer: copy it to the
		// caller's buffer the synchronous loop would have left it in
		// (the genes only: the floats past num_of_genes stay the caller's, as
		// they would in the synchronous loop)
		ADGPU_CUDA_RET(cudaMemcpy2DAsync(conf[G & 1], kGenotypeStride * 4, conf[fb], kGenotypeStride * 4,
		                                 (size_t)dp.num_of_genes * 4, n, cudaMemcpyDeviceToDevice, st), "final population");
		ADGPU_CUDA_RET(cudaMemcpyAsync(en[G & 1], en[fb], n * 4, cudaMemcpyDeviceToDevice, st), "final energies");
		ADGPU_CUDA_RET(cudaStreamSynchronize(st), "final copy");
	}
	return ADGPU_OK;
}

}  // namespace adgpu
