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
// states in the reference's order -- on one device task ring, and a run
// starts its next generation as soon as its own last task ends.  The stop
// test keeps the reference's semantics exactly: check g (before generation g)
// uses the evaluations of all runs after generation g-1, so it is taken by
// whichever pose group completes the last run's generation g-1.  Runs may
// run ahead of that decision by up to kPipeBufs-1 generations: generation g
// reads population buffer g % kPipeBufs and writes buffer (g+1) % kPipeBufs,
// which holds the result of generation g - kPipeBufs; that result is needed
// only if check g - kPipeBufs + 1 says stop, so generation g may start once
// that check has said continue.  When a check says stop, the generations
// already run past it are discarded: their evaluations are taken back off the
// per-run counters and the final population is the one the reference ends
// with.  Every run performs exactly the reference's operations on its own
// population and PRNG states (local-search entity l of run r uses the states
// of GA block r*P + l, inside its own run, because the local-search rate is
// 100 %), so populations, energies and evaluation counts are bit-identical
// to the generation-synchronous loop; only the PRNG states and the per-entity
// evaluation counters of the discarded generations differ.
#include <cuda_runtime.h>
#include <cstring>
#include <vector>

#include "adgpu_kernels.cuh"
#include "adgpu_queue.cuh"
#include "adgpu_pipeline.h"

#ifndef ADGPU_MIN_CTAS
#define ADGPU_MIN_CTAS 6
#endif

namespace adgpu {

constexpr int kPipeThreads = 128;
constexpr uint32_t kPipeRunShift = 11;         // task word: run << 11 | entity
constexpr uint32_t kPipeStop = 0x7fffffffu;    // task word that ends a worker
constexpr int kRetired = 0x40000000;           // started[r] of a retired run

__host__ __device__ constexpr uint32_t pipe_word(uint32_t run, uint32_t entity)
{
	return (run << kPipeRunShift) | entity;
}

struct PipeCtl {
	QueueCtl q;                               // ring control; q.alive = runs not retired
	int dec;                                  // checks 0 .. dec-1 have said continue
	int stop_gen;                             // -1, or the generations run (the check that said stop)
	unsigned long long parks;                 // times a run waited for a check before its next generation
	unsigned long long acc[kPipeBufs];        // per generation slot: sum over runs of the evaluations after it
	int fin[kPipeBufs];                       // per generation slot: runs that completed it
};

struct PipeArgs {
	KArgs ka;                   // tables, dockpars, PRNG states, evaluation counters
	PopBufs bufs[kPipeBufs];    // generation slot k: conf_cur/e_cur = buffer k, conf/e = buffer k+1
	TaskRing ring;
	PipeCtl* ctl;
	int* started;               // R: generations started (claimed), kRetired once retired
	int* done;                  // R: generations completed (or abandoned after a stop)
	int* comp;                  // R: generations whose evaluations are in evals_runs
	int* pending;               // R: tasks of the run's current phase not yet finished
	int* inc;                   // R * kPipeBufs: evaluations each generation slot added
	int runs, pop, nworkers;
	unsigned long long max_evals;
	unsigned int max_gens;
	int group_bytes;            // shared memory per pose group (header + scratch)
};

struct PipeHdr {
	unsigned long long pos;
	long long t_enter, t_task;       // worker accounting (rank 0; globaltimer ns)
	unsigned long long busy, ntask;
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
		if (atomicCAS(p.started + r, d, kRetired) == d && atomicSub(&p.ctl->q.alive, 1) == 1)
			ring_push_n(p.ring, kPipeStop, p.nworkers);
		return;
	}
	if (d - kPipeBufs + 1 >= vc->dec) {               // parked: check d-kPipeBufs+1 still open
		atomicAdd(&p.ctl->parks, 1ull);
		return;
	}
	if (atomicCAS(p.started + r, d, d + 1) != d) return;
	p.pending[r] = p.pop;
	__threadfence();
	ring_push1(p.ring, pipe_word((uint32_t)r, 0), p.pop);
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
	if (G.rank == 0) { H.t_enter = global_ns(); H.t_task = 0; H.busy = 0; H.ntask = 0; }
	for (;;) {
		if (G.rank == 0) {
			if (H.t_task) H.busy += (unsigned long long)(global_ns() - H.t_task);
			const int w = ring_take(p.ring);
			H.task = (w < 0 || (uint32_t)w == kPipeStop) ? -1 : w;
			H.t_task = H.task >= 0 ? global_ns() : 0;
			H.ntask += H.task >= 0;
			if (H.task >= 0) {
				H.gen = vload(p.started + (H.task >> kPipeRunShift)) - 1;
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
			const PopBufs pb = p.bufs[g & (kPipeBufs - 1)];
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
		if (G.rank == 0) H.last = (atomicSub(p.pending + run, 1) == 1);
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
			const int slot = g & (kPipeBufs - 1);
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
						if ((ev > gp ? ev : gp) >= 100.0) vc->stop_gen = g + 1;
						else vc->dec = g + 2;
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
		atomicAdd(&p.ctl->q.tasks, H.ntask);
		atomicAdd(&p.ctl->q.workers, 1);
		atomicMin(&p.ctl->q.t_first, (unsigned long long)H.t_enter);
		atomicMax(&p.ctl->q.t_last, (unsigned long long)global_ns());
	}
}

template <int TPP, int LSMET>
__global__ void __launch_bounds__(kPipeThreads, ADGPU_MIN_CTAS) pipe_kernel(const PipeArgs p)
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
		if (!stop)
			for (int e = 0; e < p.pop; e++) {
				const unsigned long long pos = (unsigned long long)r * p.pop + e;
				p.ring.slots[pos] = (1ull << 32) | pipe_word((uint32_t)r, (uint32_t)e);
			}
	}
	// nothing to run: one stop word per worker
	if (stop)
		for (int i = threadIdx.x; i < p.nworkers; i += blockDim.x) p.ring.slots[i] = (1ull << 32) | kPipeStop;
	if (threadIdx.x == 0) {
		PipeCtl* c = p.ctl;
		c->q.head = 0;
		c->q.tail = stop ? (unsigned long long)p.nworkers : (unsigned long long)p.runs * p.pop;
		c->q.alive = stop ? 0 : p.runs;
		c->dec = 1;
		c->stop_gen = stop ? 0 : -1;
		c->q.t_first = ~0ull;
	}
}

// Takes the evaluations of discarded generations back off the per-run
// counters.  out: generations run, runs not retired, ring error, most
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
			for (int k = G; k < p.comp[r]; k++) p.ka.evals_runs[r] -= p.inc[r * kPipeBufs + (k & (kPipeBufs - 1))];
			atomicMax(&past, p.done[r] - G);
		}
	__syncthreads();
	if (threadIdx.x == 0) {
		const QueueCtl& q = p.ctl->q;
		out[0] = G; out[1] = q.alive; out[2] = q.err; out[3] = past;
		out[4] = (long long)q.busy_ns; out[5] = (long long)q.tasks;
		out[6] = q.workers ? (long long)(q.t_last - q.t_first) : 0;
		out[7] = (long long)p.ctl->parks; out[8] = q.workers;
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
	const int pct = smem_carveout_pct(bytes, ADGPU_MIN_CTAS);
	if (pct >= 0) ADGPU_CUDA_RET(cudaFuncSetAttribute(kfn, cudaFuncAttributePreferredSharedMemoryCarveout, pct), "pipeline carveout");
	int per_sm = 0, dev = 0, sms = 0;
	ADGPU_CUDA_RET(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kPipeThreads, bytes), "pipeline occupancy");
	if (per_sm < 1) return fail(ADGPU_ERR_LIMIT, "pipeline kernel does not fit on an SM");
	ADGPU_CUDA_RET(cudaGetDevice(&dev), "device");
	ADGPU_CUDA_RET(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "sm count");
	const long useful = ((long)p.runs * p.pop + gpc - 1) / gpc;
	long grid = (long)per_sm * sms;
	if (grid > useful) grid = useful;
	p.nworkers = (int)grid * gpc;
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

// Threads per pose of the pipelined loop.  Solis-Wets and ADADELTA: 64.
// Their searches stop on their own test (cfg2 ADADELTA: mean 67, up to 300
// iterations), so a run's generation lasts as long as its longest search, and
// with 32 threads per pose that chain of generations, not the pose groups'
// throughput, sets the docking time (B200, cfg2 ADADELTA, 100 runs: 64
// threads 150 M evals/s with the pose groups 99 % busy, 32 threads 140 M at
// 81 % busy).  ADAM and FIRE run a fixed iteration count, so a generation
// holds far more work than its longest chain: 32, the group size with the
// higher throughput.
int pipeline_default_tpp(int lsmet)
{
	return (lsmet == 0 || lsmet == 1) ? 64 : 32;
}

adgpu_status dock_pipelined(const KArgs& base, PipeScratch& sc, int lsmet, int tpp, uint32_t runs,
                            uint64_t max_evals, uint32_t max_gens, float* c1, float* e1, float* c2, float* e2,
                            int* final_is_second, uint32_t* generations)
{
	const adgpu_dockpars& dp = base.dp;
	if (!pipeline_applies(dp, runs)) return fail(ADGPU_ERR_ARG, "pipelined docking needs a 100 % local-search rate");
	if (tpp == 0) tpp = pipeline_default_tpp(lsmet);
	if (tpp != 32 && tpp != 64 && tpp != 128) return fail(ADGPU_ERR_ARG, "threads per pose must be 32, 64 or 128");
	const int P = dp.pop_size;
	const size_t n = (size_t)runs * P;
	// in flight at once: at most one generation's tasks per run, plus one
	// claimed position and one stop word per worker (at most 148 SMs x 32
	// pose groups here; the device's count is checked below)
	int dev = 0, sms = 0;
	ADGPU_CUDA_RET(cudaGetDevice(&dev), "device");
	ADGPU_CUDA_RET(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "sm count");
	const size_t max_workers = (size_t)sms * 2048 / 32;
	const size_t cap = 2 * ((size_t)runs * P + 2 * max_workers) + 1024;
	// scratch: two more population buffers, the ring, per-run counters, control
	auto al = [](size_t b) { return (b + 255) / 256 * 256; };
	const size_t o_conf = 0, conf_b = al(n * kGenotypeStride * 4) * 2;
	const size_t o_e = o_conf + conf_b, e_b = al(n * 4) * 2;
	const size_t o_slots = o_e + e_b, slots_b = al(cap * 8);
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
	float* conf[kPipeBufs] = {c1, c2, reinterpret_cast<float*>(m + o_conf), reinterpret_cast<float*>(m + o_conf + conf_b / 2)};
	float* en[kPipeBufs] = {e1, e2, reinterpret_cast<float*>(m + o_e), reinterpret_cast<float*>(m + o_e + e_b / 2)};
	PipeArgs p;
	memset(&p, 0, sizeof(p));
	p.ka = base;
	p.ka.ref_threads = 64;
	p.ka.stop_flag = nullptr;
	p.ka.work_counter = nullptr;
	p.ka.nblocks = 0;
	p.ka.conf_cur = p.ka.e_cur = nullptr;
	p.ka.conf = p.ka.e = nullptr;
	for (int k = 0; k < kPipeBufs; k++)
		p.bufs[k] = PopBufs{conf[k], en[k], conf[(k + 1) % kPipeBufs], en[(k + 1) % kPipeBufs]};
	p.ring.slots = reinterpret_cast<unsigned long long*>(m + o_slots);
	p.ring.cap = (uint32_t)cap;
	p.ring.slot_spin = 1 << 20;     // (ring_take bounds its wait by idle_ns)
	p.ring.idle_ns = 2000000000ll;
	int* ri = reinterpret_cast<int*>(m + o_runs);
	const size_t rs = al((size_t)runs * 4) / 4;
	p.started = ri; p.done = ri + rs; p.comp = ri + 2 * rs; p.pending = ri + 3 * rs; p.inc = ri + 4 * rs;
	p.ctl = reinterpret_cast<PipeCtl*>(m + o_ctl);
	p.ring.ctl = &p.ctl->q;
	long long* d_out = reinterpret_cast<long long*>(m + o_ctl + al(sizeof(PipeCtl)));
	p.runs = (int)runs; p.pop = P;
	p.max_evals = max_evals; p.max_gens = max_gens;
	p.group_bytes = kPipeHdrBytes + group_smem_bytes(base.L.natoms, base.L.ntors, 64, tpp);

	cudaStream_t st = 0;   // the legacy stream: ordered after the caller's initial-population calls
	// the library's population buffers start as zeros, like the caller's
	// second buffer: genes past num_of_genes are never written
	ADGPU_CUDA_RET(cudaMemsetAsync(m + o_conf, 0, conf_b + e_b, st), "pipeline buffers");
	ADGPU_CUDA_RET(cudaMemsetAsync(p.ctl, 0, sizeof(PipeCtl), st), "pipeline control");
	ADGPU_CUDA_RET(cudaMemsetAsync(p.ring.slots, 0, cap * 8, st), "pipeline ring");
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
	ADGPU_CUDA_RET(cudaMemcpyAsync(sc.host_out, d_out, 9 * sizeof(long long), cudaMemcpyDeviceToHost, st), "pipeline readback");
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
	if (err != 0 || alive != 0 || G < 0)
		return fail(ADGPU_ERR_TIMEOUT, "pipelined docking: a bounded device wait gave up (ring error " + std::to_string(err) +
		                                ", runs still active " + std::to_string(alive) + ")");
	*generations = (uint32_t)G;
	*final_is_second = G & 1;
	const int fb = G & (kPipeBufs - 1);
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
