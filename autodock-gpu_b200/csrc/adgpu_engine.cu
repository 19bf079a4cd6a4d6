// adgpu_engine.cu -- the batch / serving engine (include/adgpu_b200.h, layer 2).
//
// Many docking requests (ligands of uneven size, each with its own runs)
// against device-resident receptor maps.  A request's populations, energies,
// eval counters and PRNG states live on the device from submission to
// completion.  The engine advances all admitted runs with one persistent
// kernel per local-search method whose pose groups are workers on task
// queues: every phase of a run (initial population, GA generation, local
// search) is split into independent tasks, and the group that finishes a
// phase's last task takes the eval sum and the stop test and queues the run's
// next phase -- no grid-wide synchronisation; runs are independent, as in the
// reference (one population per run).  A tick advances every run by up to
// `gens_per_tick` generations; between ticks the host retires finished
// requests and admits new ones (continuous batching).
//
// Semantics per run follow the reference kernels operation by operation; the
// one deliberate difference from docking_with_gpu is the stop test, taken
// per run (its own evaluations >= max_evals, or generations >= max_gens)
// instead of on the mean over all runs of a ligand, so that a run's result
// depends only on its own state: a request docks identically alone or in a mix.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "adgpu_kernels.cuh"
#include "adgpu_queue.cuh"
#include "adgpu_prep.h"
#include "adgpu_result.h"
#include "adgpu_tables.h"
#include "adgpu_nvtx.h"

namespace adgpu {

// Per-request device state (one per admitted request), read by the kernel.
struct ReqDev {
	KArgs a;                    // tables, dockpars, prng, evals_new (conf/e set per generation)
	float* conf[2];             // R*P*64, double buffered
	float* e[2];                // R*P
	int* evals_runs;            // R
	int* pending;               // R tasks of the run's current phase not yet done
	unsigned long long* next;   // R the run's open phase << 32 | entities handed out
	uint32_t* gen;              // R generations done
	uint8_t* cur;               // R current buffer index
	uint8_t* done;              // R run finished
	uint8_t* init;              // R initial population scored
	float* best_e;              // R best energy of the final population
	float* best_g;              // R*64 best genotype
	unsigned long long max_evals;
	unsigned int max_gens;
	int lsmet;
	int runs;
};

struct RunRef { int req; int run; };

// 128-thread CTAs, several per SM; every pose group of a CTA is an
// independent worker.
constexpr int kEngineThreads = 128;
// 5 CTAs per SM: the kernel holds all three pose-group sizes and every
// local search, and spills at the 80 registers 6 CTAs leave; at 5 it does
// not, and the 64-ligand batch sample docks 13 % faster (B200).
#ifndef ADGPU_ENGINE_MIN_CTAS
#define ADGPU_ENGINE_MIN_CTAS 5
#endif

// --------------------------------------------------------------------------
// scheduling
// --------------------------------------------------------------------------
// A run advances in steps: step 0 scores its initial population, step s >= 1
// is generation s-1.  Each step is split into one task per entity.  For a
// generation a task is the GA step that makes the entity (elitism, or
// tournaments, crossover, mutation and scoring) followed, at the reference's
// default 100 % local-search rate, by the entity's local search, both on the
// entity's own PRNG states in the reference's order; at a lower rate the
// local searches form a second phase of their own (the entity a search takes
// may be one another task makes).  A run hands out the entities of its
// current phase from one counter (phase << 32 | entities taken; phase =
// 2*step, or 2*step+1 for a separate local-search phase), kept per work item
// for the tick.  A pose group keeps taking entities of the run it served
// last and otherwise scans its class's runs for the least advanced one with
// entities left; the group that completes a phase's last task finalises it
// (eval sum, stop test) and opens the run's next phase.  No run waits for
// another, and no run's generation waits behind another run's.
struct TickRun {
	unsigned long long next;    // phase << 32 | entities taken
	int ntasks;                 // entities of the open phase (a hint for the scan)
	int limit;                  // steps at or above this one do not start in this tick
};

struct TickClass {
	QueueCtl* ctl;              // alive (runs not finished or parked this tick), err, accounting
	int w0, nw;                 // this class's work items
	int cta_end;                // this class's CTAs are [previous class's cta_end, cta_end)
	int group_bytes;            // shared memory per pose group
};

struct TickArgs {
	const ReqDev* reqs;
	const RunRef* work;
	TickRun* runs;              // per work item
	uint8_t* work_done;         // per work item: run finished (written when it retires)
	const uint32_t* prio;       // per work item: its request's rank by age (0 oldest), or null: all equal
	long long tick_ns;          // > 0: a worker takes no new task once this long after it started
	long long idle_ns;          // a worker that finds no task for this long stops and reports an error
	TickClass cls[3];           // threads per pose 32, 64, 128
};

constexpr int kScanWindow = 4096;                              // work items one scan looks at
constexpr long long kIdleNs = 2000000000ll;                    // default idle limit (2 s)

// Per-pose-group header in shared memory, ahead of the group's scratch.
struct GroupHdr {
	KArgs a;                    // the current request's arguments
	long long t_enter, t_task;           // worker accounting (rank 0 only)
	long long deadline;                  // globaltimer after which no task is taken; 0: none
	unsigned long long busy, ntask;
	int task_w, task_idx, req, last, next, cur, isum, sticky;
	unsigned int task_phase;
	float bv[4];
	int bi[4];
};
constexpr int kHdrBytes = (int)((sizeof(GroupHdr) + 15) / 16 * 16);

__device__ __forceinline__ int phase_tasks(const ReqDev& rq, unsigned int phase)
{
	return (phase & 1u) ? (int)rq.a.dp.num_of_lsentities : rq.a.dp.pop_size;
}

// The next task for this pose group (called by its first warp): work item,
// phase and entity in *w, *phase, *idx; false when the worker should stop
// (deadline, nothing left in its class, or the idle limit: error).
template <int TPP>
__device__ bool take_task(const TickArgs& t, const TickClass& C, int lane, int worker, GroupHdr& H,
                          int* w_out, unsigned int* phase_out, int* idx_out)
{
	volatile QueueCtl* vq = C.ctl;
	long long idle_since = -1;
	int backoff = 64;
	unsigned int rot = (unsigned int)worker * 2654435761u;
	for (int spins = 0; spins < (1 << 30); spins++) {
		if (H.deadline && global_ns() > H.deadline) return false;
		// the run served last, then a scan for the run with entities left that
		// has the lowest (request rank, step): with ranks, the oldest request's
		// least advanced run; without, the least advanced run
		int cand = -1;
		if (spins == 0 && H.sticky >= 0) {
			cand = H.sticky;
		} else {
			unsigned long long best = ~0ull;
			const int n = C.nw < kScanWindow ? C.nw : kScanWindow;
			const int off = C.nw <= kScanWindow ? 0 : (int)((rot + (unsigned)spins * 977u) % (unsigned)C.nw);
			for (int i = lane; i < n; i += 32) {
				int w = off + i;
				if (w >= C.nw) w -= C.nw;
				w += C.w0;
				const int4 r = __ldcv(reinterpret_cast<const int4*>(t.runs + w));
				const unsigned int taken = (unsigned int)r.x, phase = (unsigned int)r.y;
				const int step = (int)(phase >> 1);
				if (taken < (unsigned int)r.z && step < r.w) {
					const unsigned int rank = t.prio ? t.prio[w] : 0u;
					const unsigned long long key = ((unsigned long long)rank << 48) |
					                               ((unsigned long long)min(step, 0xFFFF) << 32) |
					                               (((unsigned int)w - (unsigned int)C.w0 + rot) % (unsigned int)C.nw);
					best = key < best ? key : best;
				}
			}
#pragma unroll
			for (int o = 16; o > 0; o >>= 1) {
				const unsigned long long x = __shfl_xor_sync(0xffffffffu, best, o);
				best = x < best ? x : best;
			}
			if (best != ~0ull) cand = C.w0 + (int)(((unsigned int)best - rot % (unsigned int)C.nw + (unsigned int)C.nw) %
			                                       (unsigned int)C.nw);
		}
		if (cand >= 0) {
			unsigned long long old = 0;
			int ok = 0;
			if (lane == 0) {
				const int4 r = __ldcv(reinterpret_cast<const int4*>(t.runs + cand));
				if ((unsigned int)r.x < (unsigned int)r.z && (int)((unsigned int)r.y >> 1) < r.w) {
					old = atomicAdd(&t.runs[cand].next, 1ull);
					const unsigned int phase = (unsigned int)(old >> 32), idx = (unsigned int)old;
					const ReqDev& rq = t.reqs[t.work[cand].req];
					ok = idx < (unsigned int)phase_tasks(rq, phase) && (int)(phase >> 1) < t.runs[cand].limit;
				}
			}
			ok = __shfl_sync(0xffffffffu, ok, 0);
			old = __shfl_sync(0xffffffffu, old, 0);
			if (ok) {
				__threadfence();
				*w_out = cand;
				*phase_out = (unsigned int)(old >> 32);
				*idx_out = (int)(unsigned int)old;
				return true;
			}
			if (spins == 0) continue;      // the sticky run had nothing left: scan at once
		}
		if (vq->alive <= 0) return false;
		const long long now = global_ns();
		if (idle_since < 0) idle_since = now;
		else if (now - idle_since > t.idle_ns) {
			if (lane == 0) atomicExch(&C.ctl->err, 1);
			return false;
		}
		__nanosleep(backoff);
		if (backoff < 4096) backoff *= 2;
	}
	if (lane == 0) atomicExch(&C.ctl->err, 2);
	return false;
}

template <int TPP>
__device__ int group_isum(int v, const Group<TPP>& G, GroupHdr& H)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	if constexpr (TPP == 32) {
		return v;
	} else {
		if (G.rank == 0) H.isum = 0;
		G.sync();
		if ((G.rank & 31) == 0) atomicAdd(&H.isum, v);
		G.sync();
		const int r = H.isum;
		G.sync();
		return r;
	}
}

// Lowest energy of a run's population (smallest index on ties) -> best_e, best_g.
template <int TPP>
__device__ void best_of_run(const ReqDev& rq, int run, int c, int P, const Group<TPP>& G, GroupHdr& H)
{
	const float* E = rq.e[c] + (size_t)run * P;
	float bv = FLT_MAX;
	int bi = 0;
	for (int i = G.rank; i < P; i += TPP)
		if (E[i] < bv) { bv = E[i]; bi = i; }
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		const float v2 = __shfl_xor_sync(0xffffffffu, bv, o);
		const int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
		if (v2 < bv || (v2 == bv && i2 < bi)) { bv = v2; bi = i2; }
	}
	if ((G.rank & 31) == 0) { H.bv[G.rank >> 5] = bv; H.bi[G.rank >> 5] = bi; }
	G.sync();
	if (G.rank == 0) {
		for (int w = 1; w < TPP / 32; w++)
			if (H.bv[w] < H.bv[0] || (H.bv[w] == H.bv[0] && H.bi[w] < H.bi[0])) { H.bv[0] = H.bv[w]; H.bi[0] = H.bi[w]; }
		rq.best_e[run] = H.bv[0];
	}
	G.sync();
	const float* src = rq.conf[c] + ((size_t)run * P + H.bi[0]) * kGenotypeStride;
	for (int k = G.rank; k < kGenotypeStride; k += TPP) rq.best_g[(size_t)run * kGenotypeStride + k] = src[k];
	G.sync();
}

// Opens phase `phase` of work item w (its run's counter and the tick's
// copy), or parks the run when the phase's step is past the tick's limit.
__device__ void open_phase(const TickArgs& t, const TickClass& C, const ReqDev& rq, int w, int run, unsigned int phase)
{
	const int n = phase_tasks(rq, phase);
	rq.pending[run] = n;
	t.runs[w].ntasks = n;
	__threadfence();
	atomicExch(&t.runs[w].next, (unsigned long long)phase << 32);
	if ((int)(phase >> 1) >= t.runs[w].limit) atomicSub(&C.ctl->alive, 1);      // parked until the next tick
}

template <int TPP, int LSMET>
__device__ void engine_worker(const TickArgs& t, const TickClass& C)
{
	extern __shared__ __align__(16) char smem[];
	const int local = threadIdx.x / TPP;
	char* base = smem + (size_t)local * C.group_bytes;
	GroupHdr& H = *reinterpret_cast<GroupHdr*>(base);
	char* scratch = base + kHdrBytes;
	Group<TPP> G;
	G.rank = threadIdx.x % TPP;
	G.bar_id = 1 + local;
	G.red = nullptr;
	const int worker = blockIdx.x * (kEngineThreads / TPP) + local;
	if (G.rank == 0) {
		H.req = -1; H.sticky = -1; H.t_enter = global_ns(); H.t_task = 0; H.busy = 0; H.ntask = 0;
		H.deadline = t.tick_ns > 0 ? H.t_enter + t.tick_ns : 0;
	}
	G.sync();
	for (;;) {
		if (G.rank < 32) {
			if (G.rank == 0 && H.t_task) H.busy += (unsigned long long)(global_ns() - H.t_task);
			int w = -1, idx = 0;
			unsigned int phase = 0;
			const bool got = take_task<TPP>(t, C, G.rank, worker, H, &w, &phase, &idx);
			if (G.rank == 0) {
				H.task_w = got ? w : -1;
				H.task_phase = phase;
				H.task_idx = idx;
				H.t_task = got ? global_ns() : 0;
				H.ntask += got;
				if (got) H.sticky = w;
			}
		}
		G.sync();
		const int w = H.task_w;
		if (w < 0) break;
		__threadfence();
		const unsigned int phase = H.task_phase;
		const int idx = H.task_idx;
		const RunRef rr = t.work[w];
		const ReqDev& rq = t.reqs[rr.req];
		const int run = rr.run;
		if (H.req != rr.req) {
			const int* src = reinterpret_cast<const int*>(&rq.a);
			int* dst = reinterpret_cast<int*>(&H.a);
			for (int i = G.rank; i < (int)(sizeof(KArgs) / 4); i += TPP) dst[i] = src[i];
			G.sync();
			if (G.rank == 0) H.req = rr.req;
		}
		G.sync();
		KArgs& a = H.a;
		const GroupSmem S = carve_group(scratch, a.L.natoms, a.L.ntors, 64, TPP);
		G.red = S.red;
		const int P = a.dp.pop_size;
		const int L = (int)a.dp.num_of_lsentities;
		const bool fused = L == P;
		const int c = rq.cur[run];
		if (phase == 0) {
			// step 0: the initial population's energies (cuda/kernel1.cu:26-55)
			initpop_block<TPP>(a, PopBufs{nullptr, nullptr, rq.conf[c], rq.e[c]}, (uint32_t)(run * P + idx), G, S);
		} else {
			const bool ls_phase = (phase & 1u) != 0;
			if (!ls_phase) ga_block<TPP>(a, PopBufs{rq.conf[c], rq.e[c], rq.conf[c ^ 1], rq.e[c ^ 1]},
			                             (uint32_t)(run * P + idx), G, S);
			if (ls_phase || (fused && L > 0)) {
				// local-search block run*L + idx; entity l of run r draws from
				// the PRNG states of GA block r*P + l (its own run's range: the
				// offset is zero when every entity is searched)
				if (ls_phase) {
					if (G.rank == 0) a.prng = rq.a.prng + (size_t)run * (size_t)(P - L) * 64;
					G.sync();
				}
				const PopBufs pb{nullptr, nullptr, rq.conf[c ^ 1], rq.e[c ^ 1]};
				const uint32_t b = (uint32_t)(run * L + idx);
				if constexpr (LSMET == LS_SW) sw_block<TPP>(a, pb, b, G, S);
				else if constexpr (LSMET == LS_AD) gradient_ls_block<TPP, LS_AD>(a, pb, b, G, S);
				else if constexpr (LSMET == LS_ADAM) gradient_ls_block<TPP, LS_ADAM>(a, pb, b, G, S);
				else fire_block<TPP>(a, pb, b, G, S);
				if (ls_phase) {
					if (G.rank == 0) a.prng = rq.a.prng;
					G.sync();
				}
			}
		}
		// the last task of the phase goes on to finalise it
		__threadfence();
		G.sync();
		if (G.rank == 0) H.last = (atomicSub(&rq.pending[run], 1) == 1);
		G.sync();
		if (!H.last) continue;
		__threadfence();
		// ---- phase end ----
		if (phase != 0 && (phase & 1u) == 0 && !fused && L > 0) {
			if (G.rank == 0) open_phase(t, C, rq, w, run, phase + 1);
			G.sync();
			continue;
		}
		if (phase != 0) {
			// eval sum of the run (cuda/kernel2.cu:26-52), generation count, buffer flip
			int s = 0;
			for (int i = G.rank; i < P; i += TPP) s += a.evals_new[run * P + i];
			s = group_isum<TPP>(s, G, H);
			if (G.rank == 0) {
				rq.evals_runs[run] += s;
				rq.gen[run] += 1;
				rq.cur[run] = (uint8_t)(rq.cur[run] ^ 1);
			}
		} else if (G.rank == 0) {
			rq.init[run] = 1;
			rq.evals_runs[run] = P;
		}
		// stop test (per run: its own evaluations, or its generations)
		if (G.rank == 0) {
			const bool stop = (unsigned long long)rq.evals_runs[run] >= rq.max_evals || rq.gen[run] >= rq.max_gens;
			H.next = stop ? 1 : 0;
			H.cur = rq.cur[run];
			if (stop) rq.done[run] = 1;
			else open_phase(t, C, rq, w, run, ((phase >> 1) + 1) << 1);
		}
		G.sync();
		if (H.next) {
			best_of_run<TPP>(rq, run, H.cur, P, G, H);
			if (G.rank == 0) {
				t.work_done[w] = 1;
				__threadfence();
				atomicSub(&C.ctl->alive, 1);
			}
			G.sync();
		}
	}
	if (G.rank == 0) {
		atomicAdd(&C.ctl->busy_ns, H.busy);
		atomicAdd(&C.ctl->tasks, H.ntask);
		atomicAdd(&C.ctl->workers, 1);
		atomicMin(&C.ctl->t_first, (unsigned long long)H.t_enter);
		atomicMax(&C.ctl->t_last, (unsigned long long)global_ns());
	}
}

// One kernel per local search; its CTAs are split into three ranges, one per
// threads-per-pose class, each range serving its class's runs.
template <int LSMET>
__global__ void __launch_bounds__(kEngineThreads, ADGPU_ENGINE_MIN_CTAS) engine_kernel(const TickArgs t)
{
	if ((int)blockIdx.x < t.cls[0].cta_end) engine_worker<32, LSMET>(t, t.cls[0]);
	else if ((int)blockIdx.x < t.cls[1].cta_end) engine_worker<64, LSMET>(t, t.cls[1]);
	else engine_worker<128, LSMET>(t, t.cls[2]);
}

// Tick set-up and tear-down: each work item's phase counter from its run's
// persistent state, with the tick's step limit, and back.  Runs that
// finished in an earlier tick (their request is still waiting for others)
// count as done at once; the rest are the classes' active runs.
struct ClassBounds { int start[13]; };

__global__ void __launch_bounds__(256) tick_load_kernel(const ReqDev* reqs, const RunRef* work, TickRun* runs,
                                                         uint8_t* done, int n, int steps, QueueCtl* ctl, ClassBounds cb)
{
	for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < n; w += gridDim.x * blockDim.x) {
		const ReqDev& rq = reqs[work[w].req];
		const int run = work[w].run;
		const unsigned long long v = rq.next[run];
		const unsigned int phase = (unsigned int)(v >> 32);
		const bool finished = rq.done[run] != 0;
		TickRun r;
		r.next = v;
		r.ntasks = phase_tasks(rq, phase);
		const long long lim = finished ? 0 : (long long)(phase >> 1) + steps;
		r.limit = (int)(lim > 0x3fffffffll ? 0x3fffffffll : lim);
		runs[w] = r;
		done[w] = finished ? 1 : 0;
		if (!finished) {
			int c = 0;
			while (c < 12 && w >= cb.start[c + 1]) c++;
			atomicAdd(&ctl[c].alive, 1);
		}
	}
}

__global__ void __launch_bounds__(256) tick_store_kernel(const ReqDev* reqs, const RunRef* work, const TickRun* runs, int n)
{
	for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < n; w += gridDim.x * blockDim.x)
		reqs[work[w].req].next[work[w].run] = runs[w].next;
}

// --------------------------------------------------------------------------
// host side
// --------------------------------------------------------------------------
// Each run's final population (the buffer its last generation wrote) into
// one contiguous block, the layout result processing takes.
__global__ void __launch_bounds__(256) gather_final_kernel(ReqDev d, int P, float* conf_out, float* e_out)
{
	const int run = blockIdx.x;
	const int c = d.cur[run];
	const size_t base = (size_t)run * P;
	const float* src = d.conf[c] + base * kGenotypeStride;
	float* dst = conf_out + base * kGenotypeStride;
	for (int k = threadIdx.x; k < P * kGenotypeStride; k += blockDim.x) dst[k] = src[k];
	for (int k = threadIdx.x; k < P; k += blockDim.x) e_out[base + k] = d.e[c][base + k];
}

struct Receptor {
	float* cells = nullptr;
	size_t bytes = 0;
	adgpu_dockpars grid_fields{};     // dims, spacing, num_map_atypes
	std::vector<std::string> types;
	~Receptor() { if (cells) cudaFree(cells); }
};

struct Request {
	uint64_t id = 0;
	int receptor = 0;
	int runs = 0;
	int tpp = 32;
	size_t bytes = 0;
	LigandTables tables;
	void* state = nullptr;          // one allocation for every per-request buffer
	ReqDev dev{};
	bool done = false;
	int natoms = 0, ntors = 0;
	double t_submit = 0, t_done = 0;
	// result processing inputs (host copies from the prepared ligand)
	PostLigand post;
	std::vector<uint32_t> pairs;
	adgpu_dockpars dp{};
};

static double now_s()
{
	timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

struct Engine {
	adgpu_engine_config cfg{};
	size_t budget = 0, used = 0;
	std::vector<std::unique_ptr<Receptor>> receptors;
	std::map<uint64_t, std::unique_ptr<Request>> requests;
	uint64_t next_id = 1;
	cudaStream_t stream = nullptr;
	ReqDev* d_reqs = nullptr; int d_reqs_cap = 0;
	// per-tick device buffers, grown on demand: work items, their phase
	// counters and done flags; the classes' control blocks
	RunRef* d_work = nullptr; int d_work_cap = 0;
	TickRun* d_runs = nullptr;
	uint32_t* d_prio = nullptr;   // per work item: request rank (priority 1)
	uint8_t* d_done = nullptr;
	QueueCtl* d_ctl = nullptr;
	long long idle_ns = kIdleNs;                  // a pose group's idle limit (engine configuration)
	cudaMemPool_t pool = nullptr;                 // request tables and state, kept by the pool when freed
	cudaEvent_t ev0 = nullptr, ev1 = nullptr;     // around a tick's launches
	std::vector<uint8_t> h_done;
	std::map<long, int> tpp_cache;     // size bucket -> tuned threads per pose
	adgpu_engine_stats stats{};
	std::mutex mu;
	~Engine()
	{
		for (auto& kv : requests)
			if (kv.second->state) { cudaFreeAsync(kv.second->state, stream); kv.second->state = nullptr; }
		if (stream) cudaStreamSynchronize(stream);
		requests.clear();
		receptors.clear();
		if (pool) cudaMemPoolDestroy(pool);
		if (d_reqs) cudaFree(d_reqs);
		if (d_work) cudaFree(d_work);
		if (d_ctl) cudaFree(d_ctl);
		if (ev0) cudaEventDestroy(ev0);
		if (ev1) cudaEventDestroy(ev1);
		if (stream) cudaStreamDestroy(stream);
	}
};

static size_t request_bytes(int runs, int pop, size_t tables)
{
	size_t n = (size_t)runs * pop;
	return tables + n * kGenotypeStride * 4 * 3 /* conf x2, prng */ + n * 4 * 3 /* e x2, evals_new */ +
	       (size_t)runs * (4 + 4 + 4 + 3 + 4 + 8 + kGenotypeStride * 4) + 1024;
}

// Launches the tick's kernel for local search LSMET.  Its CTAs are split
// between the three threads-per-pose classes in proportion to their work, each
// class getting no more CTAs than its runs can keep busy at once.
template <int LSMET>
static adgpu_status launch_engine(Engine& E, TickArgs t, const int* nruns, const double* weight, const int* max_tasks,
                                  const int* max_atoms, const int* max_tors)
{
	static const int tpps[3] = {32, 64, 128};
	int smem = 0;
	for (int k = 0; k < 3; k++) {
		t.cls[k].group_bytes = kHdrBytes + group_smem_bytes(max_atoms[k], max_tors[k], 64, tpps[k]);
		if (nruns[k]) smem = std::max(smem, t.cls[k].group_bytes * (kEngineThreads / tpps[k]));
	}
	auto kern = engine_kernel<LSMET>;
	if (smem > 48 * 1024) {
		cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
		if (e != cudaSuccess) return cuda_fail(e, "engine smem");
	}
	const int pct = smem_carveout_pct(smem, ADGPU_ENGINE_MIN_CTAS);
	if (pct >= 0) {
		cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
		if (e != cudaSuccess) return cuda_fail(e, "engine carveout");
	}
	int per_sm = 0, dev = 0, sms = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kEngineThreads, smem);
	if (e != cudaSuccess) return cuda_fail(e, "engine occupancy");
	if (per_sm < 1) return fail(ADGPU_ERR_LIMIT, "engine kernel does not fit on an SM");
	const int total = per_sm * sms;
	double wsum = 0;
	for (int k = 0; k < 3; k++) if (nruns[k]) wsum += weight[k];
	int end = 0;
	for (int k = 0; k < 3; k++) {
		int n = 0;
		if (nruns[k]) {
			const long useful = ((long)nruns[k] * max_tasks[k] + (kEngineThreads / tpps[k]) - 1) / (kEngineThreads / tpps[k]);
			n = (int)std::lround(total * (wsum > 0 ? weight[k] / wsum : 1.0));
			n = (int)std::max<long>(1, std::min<long>(n, useful));
		}
		end += n;
		t.cls[k].cta_end = end;
	}
	kern<<<end, kEngineThreads, smem, E.stream>>>(t);
	e = cudaGetLastError();
	if (e != cudaSuccess) return cuda_fail(e, "engine launch");
	return ADGPU_OK;
}

// Threads per pose for a ligand: the fastest of 32/64/128 on a short scoring
// benchmark of that ligand, cached per size bucket (atoms/16, pairs/256) so
// that every ligand of a bucket is scored with the same group size.
static int tune_tpp(Engine& E, Request& r);

}  // namespace adgpu

using namespace adgpu;

struct adgpu_engine_s { Engine e; };

extern "C" {

adgpu_status adgpu_engine_create(const adgpu_engine_config* cfg, adgpu_engine** out)
{
	if (!out) return fail(ADGPU_ERR_ARG, "null out");
	adgpu_engine* en = new (std::nothrow) adgpu_engine;
	if (!en) return fail(ADGPU_ERR_ARG, "out of host memory");
	Engine& E = en->e;
	if (cfg) E.cfg = *cfg;
	if (E.cfg.gens_per_tick <= 0) E.cfg.gens_per_tick = 1 << 30;
	if (E.cfg.threads_per_pose != 0 && E.cfg.threads_per_pose != -1 && E.cfg.threads_per_pose != 32 &&
	    E.cfg.threads_per_pose != 64 && E.cfg.threads_per_pose != 128) {
		delete en;
		return fail(ADGPU_ERR_ARG, "threads_per_pose must be -1, 0, 32, 64 or 128");
	}
	if (E.cfg.priority != 0 && E.cfg.priority != 1) {
		delete en;
		return fail(ADGPU_ERR_ARG, "priority must be 0 or 1");
	}
	cudaError_t e = cudaSetDevice(E.cfg.device);
	if (e != cudaSuccess) { delete en; return cuda_fail(e, "set device"); }
	size_t fr = 0, tot = 0;
	cudaMemGetInfo(&fr, &tot);
	E.budget = E.cfg.memory_budget_bytes ? E.cfg.memory_budget_bytes : (size_t)(0.8 * fr);
	e = cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking);
	if (e != cudaSuccess) { delete en; return cuda_fail(e, "stream"); }
	if (E.cfg.tick_ms < 0.0f || E.cfg.tick_ms != E.cfg.tick_ms) { delete en; return fail(ADGPU_ERR_ARG, "tick_ms must be >= 0"); }
	if (E.cfg.idle_timeout_ms < 0.0f || E.cfg.idle_timeout_ms != E.cfg.idle_timeout_ms) {
		delete en;
		return fail(ADGPU_ERR_ARG, "idle_timeout_ms must be >= 0");
	}
	if (E.cfg.idle_timeout_ms > 0.0f) E.idle_ns = (long long)(1e6 * (double)E.cfg.idle_timeout_ms);
	{
		cudaMemPoolProps props{};
		props.allocType = cudaMemAllocationTypePinned;
		props.location.type = cudaMemLocationTypeDevice;
		props.location.id = E.cfg.device;
		e = cudaMemPoolCreate(&E.pool, &props);
		if (e != cudaSuccess) { delete en; return cuda_fail(e, "engine memory pool"); }
		uint64_t keep = ~0ull;          // freed request memory stays in the pool for the next admission
		cudaMemPoolSetAttribute(E.pool, cudaMemPoolAttrReleaseThreshold, &keep);
	}
	e = cudaMalloc(&E.d_ctl, 12 * sizeof(QueueCtl));
	if (e != cudaSuccess) { delete en; return cuda_fail(e, "engine queues"); }
	*out = en;
	return ADGPU_OK;
}

void adgpu_engine_destroy(adgpu_engine* en) { delete en; }

adgpu_status adgpu_engine_add_receptor(adgpu_engine* en, const adgpu_grid* grid, int* receptor_id)
{
	if (!en || !grid || !receptor_id) return fail(ADGPU_ERR_ARG, "null argument");
	Engine& E = en->e;
	std::lock_guard<std::mutex> lk(E.mu);
	int dims[3]; double sp, org[3]; int nm;
	adgpu_grid_info(grid, dims, &sp, org, &nm);
	auto R = std::make_unique<Receptor>();
	size_t bytes = cell_grid_bytes(dims[0], dims[1], dims[2], nm);
	if (E.used + bytes > E.budget) return fail(ADGPU_ERR_BUDGET, "receptor maps exceed the engine's memory budget");
	std::vector<float> cells(bytes / sizeof(float));
	grid_cell_records(grid->g, cells.data());
	cudaError_t e = cudaMalloc(&R->cells, bytes);
	if (e != cudaSuccess) return cuda_fail(e, "receptor maps");
	e = cudaMemcpy(R->cells, cells.data(), bytes, cudaMemcpyHostToDevice);
	if (e != cudaSuccess) return cuda_fail(e, "receptor maps upload");
	R->bytes = bytes;
	adgpu_dockpars& gf = R->grid_fields;
	gf.gridsize_x = dims[0]; gf.gridsize_y = dims[1]; gf.gridsize_z = dims[2];
	gf.gridsize_x_times_y = dims[0] * dims[1];
	gf.gridsize_x_times_y_times_z = dims[0] * dims[1] * dims[2];
	gf.grid_spacing = (float)sp;
	gf.num_of_map_atypes = nm;
	E.used += bytes;
	E.receptors.push_back(std::move(R));
	*receptor_id = (int)E.receptors.size() - 1;
	return ADGPU_OK;
}

adgpu_status adgpu_engine_submit(adgpu_engine* en, const adgpu_ligand* lig, const adgpu_request_params* rp, uint64_t* request_id)
{
	adgpu::NvtxRange nvtx_range("adgpu_engine_submit");
	if (!en || !lig || !rp || !request_id) return fail(ADGPU_ERR_ARG, "null argument");
	Engine& E = en->e;
	std::lock_guard<std::mutex> lk(E.mu);
	if (rp->receptor < 0 || rp->receptor >= (int)E.receptors.size()) return fail(ADGPU_ERR_ARG, "unknown receptor");
	if (rp->lsmet < 0 || rp->lsmet > 3) return fail(ADGPU_ERR_ARG, "lsmet must be 0..3");
	const Receptor& R = *E.receptors[rp->receptor];
	const Prepared& p = lig->p;
	const adgpu_dockpars& dp = p.dockpars;
	if (dp.gridsize_x != R.grid_fields.gridsize_x || dp.gridsize_y != R.grid_fields.gridsize_y ||
	    dp.gridsize_z != R.grid_fields.gridsize_z || dp.grid_spacing != R.grid_fields.grid_spacing ||
	    dp.num_of_map_atypes != R.grid_fields.num_of_map_atypes)
		return fail(ADGPU_ERR_ARG, "ligand was prepared against a different grid than the receptor");
	const int runs = (int)(p.initpop.size() / ((size_t)dp.pop_size * kGenotypeStride));
	if (runs <= 0) return fail(ADGPU_ERR_ARG, "ligand has no runs (prepare it with num_runs > 0)");
	auto r = std::make_unique<Request>();
	PackedLigand pk;
	adgpu_status st = pack_ligand(dp, p.interintra, p.pairs.data(), p.intra, p.rotlist.data(), p.conform,
	                              p.grads.rotbonds, p.grads.rotbonds_atoms, p.grads.num_rotating_atoms_per_rotbond, pk);
	if (st != ADGPU_OK) return st;
	const size_t need = request_bytes(runs, dp.pop_size, pk.blob.size());
	if (E.used + need > E.budget) return fail(ADGPU_ERR_BUDGET, "request does not fit the engine's memory budget now");
	// one stream-ordered allocation from the engine's pool for the request's
	// tables and state (no device-wide synchronisation on admit or release)
	const size_t n = (size_t)runs * dp.pop_size;
	size_t off = 0;
	auto take = [&](size_t bytes) { size_t o = off; off = (off + bytes + 255) / 256 * 256; return o; };
	size_t o_tab = take(pk.blob.size()), o_c0 = take(n * kGenotypeStride * 4), o_c1 = take(n * kGenotypeStride * 4), o_e0 = take(n * 4),
	       o_e1 = take(n * 4), o_ev = take(n * 4), o_pr = take(n * 64 * 4), o_er = take(runs * 4), o_gen = take(runs * 4),
	       o_cur = take(runs), o_done = take(runs), o_init = take(runs), o_be = take(runs * 4),
	       o_bg = take((size_t)runs * kGenotypeStride * 4), o_pend = take((size_t)runs * 4),
	       o_next = take((size_t)runs * 8);
	cudaError_t e = cudaMallocFromPoolAsync(&r->state, off, E.pool, E.stream);
	if (e != cudaSuccess) return cuda_fail(e, "request state");
	char* B = static_cast<char*>(r->state);
	e = cudaMemsetAsync(B + o_c0, 0, off - o_c0, E.stream);
	if (e == cudaSuccess) e = cudaMemcpyAsync(B + o_tab, pk.blob.data(), pk.blob.size(), cudaMemcpyHostToDevice, E.stream);
	if (e == cudaSuccess) e = cudaMemcpyAsync(B + o_c0, p.initpop.data(), n * kGenotypeStride * 4, cudaMemcpyHostToDevice, E.stream);
	if (e == cudaSuccess) e = cudaMemcpyAsync(B + o_pr, p.prng.data(), n * 64 * 4, cudaMemcpyHostToDevice, E.stream);
	// step 0 (scoring the initial population) open: its P entities pending,
	// none handed out (the phase counters are zero from the memset)
	if (e == cudaSuccess) {
		std::vector<int> pend(runs, dp.pop_size);
		e = cudaMemcpyAsync(B + o_pend, pend.data(), (size_t)runs * 4, cudaMemcpyHostToDevice, E.stream);
		if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
	}
	if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
	if (e != cudaSuccess) { cudaFreeAsync(r->state, E.stream); r->state = nullptr; return cuda_fail(e, "request upload"); }
	place_ligand(pk, B + o_tab, r->tables.dev);
	set_grid_fields(r->tables.dev, dp, R.cells);
	r->tables.own_grid = false;
	r->tables.dgrid = nullptr;
	r->tables.packed = pk;
	ReqDev& d = r->dev;
	memset(&d, 0, sizeof(d));
	d.a.L = r->tables.dev;
	d.a.dp = dp;
	d.a.prng = reinterpret_cast<uint32_t*>(B + o_pr);
	d.a.evals_new = reinterpret_cast<int*>(B + o_ev);
	d.a.ref_threads = 64;
	d.conf[0] = reinterpret_cast<float*>(B + o_c0);
	d.conf[1] = reinterpret_cast<float*>(B + o_c1);
	d.e[0] = reinterpret_cast<float*>(B + o_e0);
	d.e[1] = reinterpret_cast<float*>(B + o_e1);
	d.evals_runs = reinterpret_cast<int*>(B + o_er);
	d.gen = reinterpret_cast<uint32_t*>(B + o_gen);
	d.cur = reinterpret_cast<uint8_t*>(B + o_cur);
	d.done = reinterpret_cast<uint8_t*>(B + o_done);
	d.init = reinterpret_cast<uint8_t*>(B + o_init);
	d.best_e = reinterpret_cast<float*>(B + o_be);
	d.best_g = reinterpret_cast<float*>(B + o_bg);
	d.pending = reinterpret_cast<int*>(B + o_pend);
	d.next = reinterpret_cast<unsigned long long*>(B + o_next);
	d.max_evals = rp->max_evals;
	d.max_gens = rp->max_gens ? rp->max_gens : 0xFFFFFFFFu;
	d.lsmet = rp->lsmet;
	d.runs = runs;
	r->id = E.next_id++;
	r->receptor = rp->receptor;
	r->runs = runs;
	r->post = lig->p.post;
	r->pairs = lig->p.pairs;
	r->dp = dp;
	r->bytes = need;
	r->natoms = dp.num_of_atoms;
	r->ntors = dp.num_of_genes - 6;
	// threads per pose: the configured size; by default one warp, the size
	// with the most evaluations per SM (runs advance independently and every
	// entity is a task of its own, so no generation waits behind a longest
	// search); -1: the fastest size on a short scoring benchmark of the
	// ligand.  (64 uneven ligands, nrun 20, ADADELTA: 100 k ligands/h with
	// 32 for all, 97 k with 64, 76 k with the tuned sizes, whose classes
	// split the GPU between them.)
	if (E.cfg.threads_per_pose > 0) r->tpp = E.cfg.threads_per_pose;
	else if (E.cfg.threads_per_pose < 0) r->tpp = tune_tpp(E, *r);
	else r->tpp = 32;
	r->t_submit = now_s();
	E.used += need;
	E.stats.submitted++;
	*request_id = r->id;
	E.requests[r->id] = std::move(r);
	return ADGPU_OK;
}

adgpu_status adgpu_engine_tick(adgpu_engine* en, int* completed)
{
	adgpu::NvtxRange nvtx_range("adgpu_engine_tick");
	if (!en) return fail(ADGPU_ERR_ARG, "null engine");
	Engine& E = en->e;
	std::lock_guard<std::mutex> lk(E.mu);
	// active requests and their runs, grouped by class = threads-per-pose index * 4 + local search
	constexpr int NC = 12;
	std::vector<ReqDev> reqs;
	std::vector<Request*> order;
	std::vector<RunRef> work[NC];
	int max_atoms[NC], max_tors[NC], max_tasks[NC];
	double weight[NC];
	for (int c = 0; c < NC; c++) { max_atoms[c] = 1; max_tors[c] = 0; max_tasks[c] = 1; weight[c] = 0; }
	std::vector<uint32_t> wprio[NC];      // request rank by age (E.requests is ordered by id = admission)
	for (auto& kv : E.requests) {
		Request& r = *kv.second;
		if (r.done) continue;
		const int cls = (r.tpp == 32 ? 0 : (r.tpp == 64 ? 1 : 2)) * 4 + r.dev.lsmet;
		const int idx = (int)reqs.size();
		reqs.push_back(r.dev);
		order.push_back(&r);
		for (int k = 0; k < r.runs; k++) {
			work[cls].push_back({idx, k});
			wprio[cls].push_back((uint32_t)std::min(idx, 0xFFFF));
		}
		const adgpu_dockpars& dp = r.dev.a.dp;
		max_atoms[cls] = std::max(max_atoms[cls], r.natoms);
		max_tors[cls] = std::max(max_tors[cls], r.ntors);
		max_tasks[cls] = std::max({max_tasks[cls], (int)dp.num_of_lsentities, dp.pop_size});
		weight[cls] += (double)r.runs * (r.dev.a.L.npairs + 8.0 * r.natoms + 64.0);
	}
	if (completed) *completed = 0;
	if (reqs.empty()) return ADGPU_OK;
	size_t start[NC];
	std::vector<RunRef> all;
	std::vector<uint32_t> all_prio;
	for (int c = 0; c < NC; c++) {
		start[c] = all.size();
		all.insert(all.end(), work[c].begin(), work[c].end());
		all_prio.insert(all_prio.end(), wprio[c].begin(), wprio[c].end());
	}
	const size_t nwork = all.size();
	if (nwork >= (size_t)0x3fffffff) return fail(ADGPU_ERR_LIMIT, "too many runs admitted at once");
	cudaError_t e;
	if ((int)reqs.size() > E.d_reqs_cap) {
		if (E.d_reqs) cudaFree(E.d_reqs);
		E.d_reqs_cap = std::max<int>((int)reqs.size() * 2, 64);
		e = cudaMalloc(&E.d_reqs, sizeof(ReqDev) * E.d_reqs_cap);
		if (e != cudaSuccess) { E.d_reqs = nullptr; E.d_reqs_cap = 0; return cuda_fail(e, "request table"); }
	}
	if ((int)nwork > E.d_work_cap) {
		if (E.d_work) cudaFree(E.d_work);
		E.d_work_cap = std::max<int>((int)nwork * 2, 256);
		const size_t per = sizeof(RunRef) + sizeof(TickRun) + 1 + sizeof(uint32_t);
		e = cudaMalloc(&E.d_work, per * E.d_work_cap + 256);
		if (e != cudaSuccess) { E.d_work = nullptr; E.d_work_cap = 0; return cuda_fail(e, "work list"); }
		char* B = reinterpret_cast<char*>(E.d_work) + sizeof(RunRef) * E.d_work_cap;
		B = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(B) + 15) & ~uintptr_t(15));
		E.d_runs = reinterpret_cast<TickRun*>(B);
		E.d_prio = reinterpret_cast<uint32_t*>(E.d_runs + E.d_work_cap);
		E.d_done = reinterpret_cast<uint8_t*>(E.d_prio + E.d_work_cap);
	}
	QueueCtl h_ctl[NC];
	memset(h_ctl, 0, sizeof(h_ctl));
	ClassBounds cb;
	for (int c = 0; c < NC; c++) {
		h_ctl[c].alive = 0;                  // counted by tick_load_kernel
		h_ctl[c].t_first = ~0ull;
		cb.start[c] = (int)start[c];
	}
	cb.start[NC] = (int)nwork;
	e = cudaMemcpyAsync(E.d_reqs, reqs.data(), sizeof(ReqDev) * reqs.size(), cudaMemcpyHostToDevice, E.stream);
	if (e == cudaSuccess) e = cudaMemcpyAsync(E.d_work, all.data(), sizeof(RunRef) * nwork, cudaMemcpyHostToDevice, E.stream);
	if (e == cudaSuccess && E.cfg.priority == 1)
		e = cudaMemcpyAsync(E.d_prio, all_prio.data(), sizeof(uint32_t) * nwork, cudaMemcpyHostToDevice, E.stream);
	if (e == cudaSuccess) e = cudaMemcpyAsync(E.d_ctl, h_ctl, sizeof(h_ctl), cudaMemcpyHostToDevice, E.stream);
	if (e != cudaSuccess) return cuda_fail(e, "tick upload");
	const int lgrid = (int)std::min<size_t>((nwork + 255) / 256, 1024);
	tick_load_kernel<<<lgrid, 256, 0, E.stream>>>(E.d_reqs, E.d_work, E.d_runs, E.d_done, (int)nwork, E.cfg.gens_per_tick,
	                                              E.d_ctl, cb);
	e = cudaGetLastError();
	if (e != cudaSuccess) return cuda_fail(e, "tick load");
	if (!E.ev0) { cudaEventCreate(&E.ev0); cudaEventCreate(&E.ev1); }
	cudaEventRecord(E.ev0, E.stream);
	for (int m = 0; m < 4; m++) {
		int nr[3], ma[3], mt[3], mx[3];
		double wt[3];
		bool any = false;
		TickArgs t;
		memset(&t, 0, sizeof(t));
		t.reqs = E.d_reqs; t.work = E.d_work; t.runs = E.d_runs; t.work_done = E.d_done;
		t.prio = E.cfg.priority == 1 ? E.d_prio : nullptr;
		t.tick_ns = (long long)(1e6 * (double)E.cfg.tick_ms);
		t.idle_ns = E.idle_ns;
		for (int k = 0; k < 3; k++) {
			const int c = k * 4 + m;
			nr[k] = (int)work[c].size(); ma[k] = max_atoms[c]; mt[k] = max_tors[c]; mx[k] = max_tasks[c]; wt[k] = weight[c];
			t.cls[k].ctl = E.d_ctl + c;
			t.cls[k].w0 = (int)start[c];
			t.cls[k].nw = nr[k];
			any |= nr[k] > 0;
		}
		if (!any) continue;
		adgpu_status st = ADGPU_OK;
		switch (m) {
		case LS_SW: st = launch_engine<LS_SW>(E, t, nr, wt, mx, ma, mt); break;
		case LS_AD: st = launch_engine<LS_AD>(E, t, nr, wt, mx, ma, mt); break;
		case LS_ADAM: st = launch_engine<LS_ADAM>(E, t, nr, wt, mx, ma, mt); break;
		default: st = launch_engine<LS_FIRE>(E, t, nr, wt, mx, ma, mt); break;
		}
		if (st != ADGPU_OK) return st;
	}
	cudaEventRecord(E.ev1, E.stream);
	// the runs' phase counters back into their requests' state: a phase
	// begun in this tick continues in the next
	tick_store_kernel<<<lgrid, 256, 0, E.stream>>>(E.d_reqs, E.d_work, E.d_runs, (int)nwork);
	e = cudaGetLastError();
	if (e != cudaSuccess) return cuda_fail(e, "tick store");
	E.h_done.resize(nwork);
	e = cudaMemcpyAsync(E.h_done.data(), E.d_done, nwork, cudaMemcpyDeviceToHost, E.stream);
	if (e == cudaSuccess) e = cudaMemcpyAsync(h_ctl, E.d_ctl, sizeof(h_ctl), cudaMemcpyDeviceToHost, E.stream);
	if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
	if (e != cudaSuccess) return cuda_fail(e, "engine tick");
	const bool timed = E.cfg.tick_ms > 0.0f;
	for (int c = 0; c < NC; c++) {
		if (h_ctl[c].err)
			return fail(ADGPU_ERR_TIMEOUT, "engine tick: pose groups found no task for the idle limit while runs were "
			                               "still active (a phase whose tasks never completed)");
		if (h_ctl[c].alive != 0 && !timed) return fail(ADGPU_ERR_STATE, "engine tick ended with runs still active");
		if (h_ctl[c].workers > 0 && h_ctl[c].t_last > h_ctl[c].t_first) {
			E.stats.worker_busy_s += 1e-9 * (double)h_ctl[c].busy_ns;
			E.stats.worker_span_s += 1e-9 * (double)h_ctl[c].workers * (double)(h_ctl[c].t_last - h_ctl[c].t_first);
			E.stats.tasks += h_ctl[c].tasks;
		}
	}
	float kms = 0.0f;
	if (cudaEventElapsedTime(&kms, E.ev0, E.ev1) == cudaSuccess) E.stats.kernel_s += 1e-3 * kms;
	E.stats.ticks++;
	// a request is complete when all its runs are
	std::vector<int> runs_done(order.size(), 0);
	for (size_t i = 0; i < nwork; i++)
		if (E.h_done[i]) runs_done[all[i].req]++;
	int comp = 0;
	double tnow = now_s();
	for (size_t i = 0; i < order.size(); i++)
		if (runs_done[i] == order[i]->runs) {
			order[i]->done = true;
			order[i]->t_done = tnow;
			comp++;
		}
	E.stats.completed += comp;
	if (completed) *completed = comp;
	return ADGPU_OK;
}

adgpu_status adgpu_engine_cancel(adgpu_engine* en, uint64_t request_id)
{
	if (!en) return fail(ADGPU_ERR_ARG, "null engine");
	Engine& E = en->e;
	std::lock_guard<std::mutex> lk(E.mu);
	auto it = E.requests.find(request_id);
	if (it == E.requests.end()) return fail(ADGPU_ERR_ARG, "unknown request");
	Request& r = *it->second;
	if (r.state) cudaFreeAsync(r.state, E.stream);
	r.state = nullptr;
	E.used -= r.bytes;
	E.stats.cancelled++;
	E.requests.erase(it);
	return ADGPU_OK;
}

adgpu_status adgpu_engine_inject_stall(adgpu_engine* en, uint64_t request_id)
{
	if (!en) return fail(ADGPU_ERR_ARG, "null engine");
	Engine& E = en->e;
	std::lock_guard<std::mutex> lk(E.mu);
	auto it = E.requests.find(request_id);
	if (it == E.requests.end()) return fail(ADGPU_ERR_ARG, "unknown request");
	Request& r = *it->second;
	if (r.done) return fail(ADGPU_ERR_STATE, "request already finished");
	// every entity of each run's open phase handed out, none completed
	std::vector<unsigned long long> next(r.runs);
	cudaError_t e = cudaMemcpyAsync(next.data(), r.dev.next, (size_t)r.runs * 8, cudaMemcpyDeviceToHost, E.stream);
	if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
	if (e != cudaSuccess) return cuda_fail(e, "stall read");
	for (auto& v : next) v = (v & 0xffffffff00000000ull) | 0xffffffull;
	e = cudaMemcpyAsync(r.dev.next, next.data(), (size_t)r.runs * 8, cudaMemcpyHostToDevice, E.stream);
	if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
	return e == cudaSuccess ? ADGPU_OK : cuda_fail(e, "stall write");
}

adgpu_status adgpu_engine_run(adgpu_engine* en)
{
	if (!en) return fail(ADGPU_ERR_ARG, "null engine");
	for (;;) {
		bool active = false;
		{
			std::lock_guard<std::mutex> lk(en->e.mu);
			for (auto& kv : en->e.requests) if (!kv.second->done) { active = true; break; }
		}
		if (!active) return ADGPU_OK;
		int c = 0;
		adgpu_status st = adgpu_engine_tick(en, &c);
		if (st != ADGPU_OK) return st;
	}
}

adgpu_status adgpu_engine_poll(adgpu_engine* en, uint64_t request_id, int* done)
{
	if (!en || !done) return fail(ADGPU_ERR_ARG, "null argument");
	std::lock_guard<std::mutex> lk(en->e.mu);
	auto it = en->e.requests.find(request_id);
	if (it == en->e.requests.end()) return fail(ADGPU_ERR_ARG, "unknown request");
	*done = it->second->done ? 1 : 0;
	return ADGPU_OK;
}

adgpu_status adgpu_engine_result(adgpu_engine* en, uint64_t request_id, float* best_energies, float* best_genotypes,
                                 int* evals, uint32_t* generations, double* latency_s)
{
	if (!en) return fail(ADGPU_ERR_ARG, "null engine");
	Engine& E = en->e;
	std::lock_guard<std::mutex> lk(E.mu);
	auto it = E.requests.find(request_id);
	if (it == E.requests.end()) return fail(ADGPU_ERR_ARG, "unknown request");
	Request& r = *it->second;
	if (!r.done) return fail(ADGPU_ERR_STATE, "request still running");
	cudaError_t e = cudaSuccess;
	if (best_energies) e = cudaMemcpy(best_energies, r.dev.best_e, r.runs * 4, cudaMemcpyDeviceToHost);
	if (e == cudaSuccess && best_genotypes)
		e = cudaMemcpy(best_genotypes, r.dev.best_g, (size_t)r.runs * kGenotypeStride * 4, cudaMemcpyDeviceToHost);
	if (e == cudaSuccess && evals) e = cudaMemcpy(evals, r.dev.evals_runs, r.runs * 4, cudaMemcpyDeviceToHost);
	if (e == cudaSuccess && generations) e = cudaMemcpy(generations, r.dev.gen, r.runs * 4, cudaMemcpyDeviceToHost);
	if (e != cudaSuccess) return cuda_fail(e, "result download");
	if (latency_s) *latency_s = r.t_done - r.t_submit;
	// release the request's device memory: its slots are free for new admissions
	if (r.state) cudaFreeAsync(r.state, E.stream);
	r.state = nullptr;
	E.used -= r.bytes;
	E.requests.erase(it);
	return ADGPU_OK;
}

adgpu_status adgpu_engine_process_result(adgpu_engine* en, uint64_t request_id, const adgpu_result_params* params,
                                         adgpu_run_result* runs, adgpu_cluster* clusters, int* num_clusters,
                                         double* best_xyz, float* peratom, float* entities, float* final_population,
                                         float* final_energies)
{
	adgpu::NvtxRange nvtx_range("adgpu_engine_process_result");
	if (!en || !params) return fail(ADGPU_ERR_ARG, "null argument");
	Engine& E = en->e;
	std::lock_guard<std::mutex> lk(E.mu);
	auto it = E.requests.find(request_id);
	if (it == E.requests.end()) return fail(ADGPU_ERR_ARG, "unknown request");
	Request& r = *it->second;
	if (!r.done) return fail(ADGPU_ERR_STATE, "request still running");
	const Receptor& R = *E.receptors[r.receptor];
	const int P = r.dp.pop_size;
	const size_t npop = (size_t)r.runs * P;
	void* scratch = nullptr;
	cudaError_t e = cudaMallocFromPoolAsync(&scratch, npop * (kGenotypeStride + 1) * 4, E.pool, E.stream);
	if (e != cudaSuccess) return cuda_fail(e, "result gather");
	float* conf = static_cast<float*>(scratch);
	float* en_ = conf + npop * kGenotypeStride;
	gather_final_kernel<<<r.runs, 256, 0, E.stream>>>(r.dev, P, conf, en_);
	adgpu_status st = process_result_core(r.post, r.pairs.data(), r.dp, R.cells, 1, conf, en_, (uint32_t)r.runs, params,
	                                      runs, clusters, num_clusters, best_xyz, peratom, entities, E.stream, E.pool);
	if (st == ADGPU_OK && final_population)
		e = cudaMemcpyAsync(final_population, conf, npop * kGenotypeStride * 4, cudaMemcpyDeviceToHost, E.stream);
	if (st == ADGPU_OK && e == cudaSuccess && final_energies)
		e = cudaMemcpyAsync(final_energies, en_, npop * 4, cudaMemcpyDeviceToHost, E.stream);
	cudaFreeAsync(scratch, E.stream);
	cudaError_t e2 = cudaStreamSynchronize(E.stream);
	if (st != ADGPU_OK) return st;
	if (e == cudaSuccess) e = e2;
	return e == cudaSuccess ? ADGPU_OK : cuda_fail(e, "result download");
}

adgpu_status adgpu_engine_stats_get(adgpu_engine* en, adgpu_engine_stats* out)
{
	if (!en || !out) return fail(ADGPU_ERR_ARG, "null argument");
	std::lock_guard<std::mutex> lk(en->e.mu);
	*out = en->e.stats;
	out->bytes_used = en->e.used;
	out->bytes_budget = en->e.budget;
	int active = 0;
	for (auto& kv : en->e.requests) active += !kv.second->done;
	out->active = active;
	return ADGPU_OK;
}

adgpu_status adgpu_engine_request_info(adgpu_engine* en, uint64_t request_id, int* threads_per_pose, int* runs)
{
	if (!en) return fail(ADGPU_ERR_ARG, "null engine");
	std::lock_guard<std::mutex> lk(en->e.mu);
	auto it = en->e.requests.find(request_id);
	if (it == en->e.requests.end()) return fail(ADGPU_ERR_ARG, "unknown request");
	if (threads_per_pose) *threads_per_pose = it->second->tpp;
	if (runs) *runs = it->second->runs;
	return ADGPU_OK;
}

}  // extern "C"

namespace adgpu {

// Scores the request's poses with each group size and keeps the fastest;
// cached per (atoms/16, pairs/256) bucket.  Every pose is scored kTuneReps
// times by a grid that fills the GPU, so the timing is the steady-state
// throughput the engine sees, not the tail of one pass over a few thousand
// poses (repeated scorings of a pose write the same values).
constexpr uint32_t kTuneReps = 8;
template <int TPP>
__global__ void __launch_bounds__(128) tune_kernel(KArgs a, float* grads)
{
	int gid, ngroups;
	Group<TPP> G;
	GroupSmem S;
	group_of<TPP>(a, gid, ngroups, G, S);
	for (uint32_t i = gid; i < kTuneReps * a.nblocks; i += ngroups) score_block<TPP, true>(a, i % a.nblocks, G, S, grads);
}

template <int TPP>
static float time_tpp(Engine& E, const KArgs& a, float* grads)
{
	const int gpc = 128 / TPP;
	const int bytes = group_smem_bytes(a.L.natoms, a.L.ntors, 64, TPP) * gpc;
	auto k = tune_kernel<TPP>;
	if (bytes > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
	int per_sm = 0, dev = 0, sms = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 128, bytes);
	if (per_sm < 1) return 1e30f;
	int grid = std::min<int>((int)((kTuneReps * a.nblocks + gpc - 1) / gpc), per_sm * sms);
	cudaEvent_t t0, t1;
	cudaEventCreate(&t0);
	cudaEventCreate(&t1);
	k<<<grid, 128, bytes, E.stream>>>(a, grads);     // warm-up
	cudaEventRecord(t0, E.stream);
	k<<<grid, 128, bytes, E.stream>>>(a, grads);
	cudaEventRecord(t1, E.stream);
	cudaEventSynchronize(t1);
	float ms = 1e30f;
	if (cudaGetLastError() == cudaSuccess) cudaEventElapsedTime(&ms, t0, t1);
	cudaEventDestroy(t0);
	cudaEventDestroy(t1);
	return ms;
}

static int tune_tpp(Engine& E, Request& r)
{
	const LigDev& L = r.tables.dev;
	long key = (long)(L.natoms / 16) * 1000 + L.npairs / 256;
	auto it = E.tpp_cache.find(key);
	if (it != E.tpp_cache.end()) return it->second;
	// poses: the request's initial population, scored with gradients
	const int n = std::min(4096, r.runs * r.dev.a.dp.pop_size);
	KArgs a;
	memset(&a, 0, sizeof(a));
	a.L = L;
	a.dp = r.dev.a.dp;
	a.conf = r.dev.conf[0];
	a.e = r.dev.e[1];
	a.ref_threads = 64;
	a.nblocks = (uint32_t)n;
	float* grads = r.dev.conf[1];
	float t32 = time_tpp<32>(E, a, grads), t64 = time_tpp<64>(E, a, grads), t128 = time_tpp<128>(E, a, grads);
	int best = 32;
	float bt = t32;
	if (t64 < bt) { bt = t64; best = 64; }
	if (t128 < bt) { bt = t128; best = 128; }
	cudaMemsetAsync(r.dev.conf[1], 0, (size_t)n * kGenotypeStride * 4, E.stream);
	cudaMemsetAsync(r.dev.e[1], 0, (size_t)n * 4, E.stream);
	cudaStreamSynchronize(E.stream);
	E.tpp_cache[key] = best;
	return best;
}

}  // namespace adgpu
