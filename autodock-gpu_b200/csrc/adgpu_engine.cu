// adgpu_engine.cu -- the batch / serving engine (include/adgpu_b200.h, layer 2).
//
// Many docking requests (ligands of uneven size, each with its own runs)
// against device-resident receptor maps.  A request's populations, energies,
// eval counters and PRNG states live on the device from submission to
// completion.  The engine advances all admitted runs with one persistent
// kernel per threads-per-pose class: a CTA takes a run from a work list and
// carries it through whole generations (initial population, GA, local
// search, eval sum, stop test) with no grid-wide synchronisation -- runs are
// independent, as in the reference (one population per run).  A tick
// advances every run by up to `gens_per_tick` generations; between ticks the
// host retires finished requests and admits new ones (continuous batching).
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
#include "adgpu_prep.h"
#include "adgpu_tables.h"

namespace adgpu {

// Per-request device state (one per admitted request), read by the kernel.
struct ReqDev {
	KArgs a;                    // tables, dockpars, prng, evals_new (conf/e set per generation)
	float* conf[2];             // R*P*64, double buffered
	float* e[2];                // R*P
	int* evals_runs;            // R
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

// 128-thread CTAs, several per SM: a CTA waits at the end of a generation's
// local search for its slowest entity, and other CTAs' runs fill the SM then.
constexpr int kEngineThreads = 128;
#ifndef ADGPU_ENGINE_MIN_CTAS
#define ADGPU_ENGINE_MIN_CTAS 6
#endif

// --------------------------------------------------------------------------
// the engine kernel (one instantiation per threads-per-pose x local search)
// --------------------------------------------------------------------------
template <int TPP, int LSMET>
__global__ void __launch_bounds__(kEngineThreads, ADGPU_ENGINE_MIN_CTAS)
engine_kernel(const ReqDev* __restrict__ reqs, const RunRef* __restrict__ work, uint8_t* work_done, int nwork, int gens_per_tick,
              unsigned int* counter, int max_atoms, int max_tors)
{
	extern __shared__ __align__(16) char smem[];
	__shared__ KArgs sa;
	__shared__ int s_item, s_ls, s_done, s_evsum;
	__shared__ float s_bv[kEngineThreads / 32];
	__shared__ int s_bi[kEngineThreads / 32];
	const int gpc = kEngineThreads / TPP, local = threadIdx.x / TPP;
	const int bytes = group_smem_bytes(max_atoms, max_tors, 64, TPP);
	GroupSmem S = carve_group(smem + local * bytes, max_atoms, max_tors, 64, TPP);
	Group<TPP> G;
	G.rank = threadIdx.x % TPP;
	G.bar_id = 1 + local;
	G.red = S.red;
	for (;;) {
		if (threadIdx.x == 0) s_item = (int)atomicAdd(counter, 1u);
		__syncthreads();
		const int item = s_item;
		if (item >= nwork) break;
		const RunRef rr = work[item];
		const ReqDev& rq = reqs[rr.req];
		const int run = rr.run;
		if (threadIdx.x == 0) sa = rq.a;
		__syncthreads();
		// the scratch of a pose group is carved for the class maximum; re-carve
		// for this ligand's sizes so offsets match what the block functions expect
		S = carve_group(smem + local * bytes, sa.L.natoms, sa.L.ntors, 64, TPP);
		G.red = S.red;
		const int P = sa.dp.pop_size;
		const uint32_t L = sa.dp.num_of_lsentities;
		for (int g = 0; g < gens_per_tick; g++) {
			if (threadIdx.x == 0) {
				int d = rq.done[run];
				if (!d && rq.init[run] &&
				    ((unsigned long long)rq.evals_runs[run] >= rq.max_evals || rq.gen[run] >= rq.max_gens)) {
					d = 1;
					rq.done[run] = 1;
				}
				s_done = d;
				s_ls = 0;
				s_evsum = 0;
			}
			__syncthreads();
			if (s_done) break;
			const int c = rq.cur[run];
			if (!rq.init[run]) {
				// initial population of this run (cuda/kernel1.cu:26-55)
				if (threadIdx.x == 0) { sa.conf = rq.conf[c]; sa.e = rq.e[c]; }
				__syncthreads();
				for (int e = local; e < P; e += gpc) initpop_block<TPP>(sa, (uint32_t)(run * P + e), G, S);
				__syncthreads();
				if (threadIdx.x == 0) { rq.init[run] = 1; rq.evals_runs[run] = P; }
				__syncthreads();
				continue;
			}
			// GA generation (cuda/kernel4.cu): current -> next
			{
				if (threadIdx.x == 0) {
					sa.conf_cur = rq.conf[c]; sa.e_cur = rq.e[c];
					sa.conf = rq.conf[c ^ 1]; sa.e = rq.e[c ^ 1];
				}
				__syncthreads();
				for (int e = local; e < P; e += gpc) ga_block<TPP>(sa, (uint32_t)(run * P + e), G, S);
			}
			__syncthreads();
			// local search on the next population, entities taken dynamically
			if (sa.dp.lsearch_rate != 0.0f) {
				const KArgs& a = sa;          // conf/e already point at the next population
				for (;;) {
					uint32_t l = 0;
					if (G.rank == 0) l = (uint32_t)atomicAdd(&s_ls, 1);
					if constexpr (TPP == 32) l = __shfl_sync(0xffffffffu, l, 0);
					else {
						if (G.rank == 0) S.misc[14] = (int)l;
						G.sync();
						l = (uint32_t)S.misc[14];
						G.sync();
					}
					if (l >= L) break;
					const uint32_t b = (uint32_t)run * L + l;
					if constexpr (LSMET == LS_SW) sw_block<TPP>(a, b, G, S);
					else if constexpr (LSMET == LS_AD) gradient_ls_block<TPP, LS_AD>(a, b, G, S);
					else if constexpr (LSMET == LS_ADAM) gradient_ls_block<TPP, LS_ADAM>(a, b, G, S);
					else fire_block<TPP>(a, b, G, S);
				}
			}
			__syncthreads();
			// eval sum of the run (cuda/kernel2.cu:26-52), generation count, buffer flip
			{
				int s = 0;
				for (int i = threadIdx.x; i < P; i += kEngineThreads) s += sa.evals_new[run * P + i];
				for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
				if ((threadIdx.x & 31) == 0) atomicAdd(&s_evsum, s);
			}
			__syncthreads();
			if (threadIdx.x == 0) {
				rq.evals_runs[run] += s_evsum;
				rq.gen[run] += 1;
				rq.cur[run] = (uint8_t)(c ^ 1);
			}
			__syncthreads();
		}
		// stop test once more, so a run that used its budget in this tick is
		// reported done now rather than at the start of the next tick
		__syncthreads();
		if (threadIdx.x == 0 && !rq.done[run] && rq.init[run] &&
		    ((unsigned long long)rq.evals_runs[run] >= rq.max_evals || rq.gen[run] >= rq.max_gens))
			rq.done[run] = 1;
		__syncthreads();
		// best member of a finished run's final population
		if (rq.done[run]) {
			const int c = rq.cur[run];
			const float* E = rq.e[c] + (size_t)run * P;
			float bv = FLT_MAX;
			int bi = 0;
			for (int i = threadIdx.x; i < P; i += kEngineThreads)
				if (E[i] < bv) { bv = E[i]; bi = i; }
			for (int o = 16; o > 0; o >>= 1) {
				float v2 = __shfl_xor_sync(0xffffffffu, bv, o);
				int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
				if (v2 < bv || (v2 == bv && i2 < bi)) { bv = v2; bi = i2; }
			}
			if ((threadIdx.x & 31) == 0) { s_bv[threadIdx.x >> 5] = bv; s_bi[threadIdx.x >> 5] = bi; }
			__syncthreads();
			if (threadIdx.x == 0) {
				for (int w = 1; w < kEngineThreads / 32; w++)
					if (s_bv[w] < s_bv[0] || (s_bv[w] == s_bv[0] && s_bi[w] < s_bi[0])) { s_bv[0] = s_bv[w]; s_bi[0] = s_bi[w]; }
				rq.best_e[run] = s_bv[0];
			}
			__syncthreads();
			const float* src = rq.conf[c] + ((size_t)run * P + s_bi[0]) * kGenotypeStride;
			for (int k = threadIdx.x; k < kGenotypeStride; k += kEngineThreads) rq.best_g[(size_t)run * kGenotypeStride + k] = src[k];
		}
		if (threadIdx.x == 0) work_done[item] = rq.done[run];
		__syncthreads();
	}
}

// --------------------------------------------------------------------------
// host side
// --------------------------------------------------------------------------
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
	RunRef* d_work = nullptr; int d_work_cap = 0;
	unsigned int* d_counters = nullptr;
	std::vector<uint8_t> h_done;
	std::map<long, int> tpp_cache;     // size bucket -> tuned threads per pose
	adgpu_engine_stats stats{};
	std::mutex mu;
	~Engine()
	{
		requests.clear();
		receptors.clear();
		if (d_reqs) cudaFree(d_reqs);
		if (d_work) cudaFree(d_work);
		if (d_counters) cudaFree(d_counters);
		if (stream) cudaStreamDestroy(stream);
	}
};

static size_t request_bytes(int runs, int pop, size_t tables)
{
	size_t n = (size_t)runs * pop;
	return tables + n * kGenotypeStride * 4 * 3 /* conf x2, prng */ + n * 4 * 3 /* e x2, evals_new */ +
	       (size_t)runs * (4 + 4 + 3 + 4 + kGenotypeStride * 4) + 1024;
}

template <int TPP, int LSMET>
static adgpu_status launch_engine(Engine& E, const RunRef* work, uint8_t* work_done, int nwork, int gens, int max_atoms, int max_tors, unsigned int* counter)
{
	const int bytes = group_smem_bytes(max_atoms, max_tors, 64, TPP) * (kEngineThreads / TPP);
	auto k = engine_kernel<TPP, LSMET>;
	if (bytes > 48 * 1024) {
		cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
		if (e != cudaSuccess) return cuda_fail(e, "engine smem");
	}
	int per_sm = 0, dev = 0, sms = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kEngineThreads, bytes);
	if (e != cudaSuccess) return cuda_fail(e, "engine occupancy");
	if (per_sm < 1) return fail(ADGPU_ERR_LIMIT, "engine kernel does not fit on an SM");
	int grid = std::min(nwork, per_sm * sms);
	k<<<grid, kEngineThreads, bytes, E.stream>>>(E.d_reqs, work, work_done, nwork, gens, counter, max_atoms, max_tors);
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
	if (E.cfg.threads_per_pose != 0 && E.cfg.threads_per_pose != 32 && E.cfg.threads_per_pose != 64 &&
	    E.cfg.threads_per_pose != 128) { delete en; return fail(ADGPU_ERR_ARG, "threads_per_pose must be 0, 32, 64 or 128"); }
	cudaError_t e = cudaSetDevice(E.cfg.device);
	if (e != cudaSuccess) { delete en; return cuda_fail(e, "set device"); }
	size_t fr = 0, tot = 0;
	cudaMemGetInfo(&fr, &tot);
	E.budget = E.cfg.memory_budget_bytes ? E.cfg.memory_budget_bytes : (size_t)(0.8 * fr);
	e = cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking);
	if (e != cudaSuccess) { delete en; return cuda_fail(e, "stream"); }
	e = cudaMalloc(&E.d_counters, 64 * sizeof(unsigned int));
	if (e != cudaSuccess) { delete en; return cuda_fail(e, "engine counters"); }
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
	st = upload_ligand(pk, r->tables);
	if (st != ADGPU_OK) return st;
	set_grid_fields(r->tables.dev, dp, R.cells);
	r->tables.own_grid = false;
	r->tables.dgrid = nullptr;
	// one allocation for the request's state
	const size_t n = (size_t)runs * dp.pop_size;
	size_t off = 0;
	auto take = [&](size_t bytes) { size_t o = off; off = (off + bytes + 255) / 256 * 256; return o; };
	size_t o_c0 = take(n * kGenotypeStride * 4), o_c1 = take(n * kGenotypeStride * 4), o_e0 = take(n * 4),
	       o_e1 = take(n * 4), o_ev = take(n * 4), o_pr = take(n * 64 * 4), o_er = take(runs * 4), o_gen = take(runs * 4),
	       o_cur = take(runs), o_done = take(runs), o_init = take(runs), o_be = take(runs * 4),
	       o_bg = take((size_t)runs * kGenotypeStride * 4);
	cudaError_t e = cudaMalloc(&r->state, off);
	if (e != cudaSuccess) return cuda_fail(e, "request state");
	char* B = static_cast<char*>(r->state);
	e = cudaMemsetAsync(B, 0, off, E.stream);
	if (e == cudaSuccess) e = cudaMemcpyAsync(B + o_c0, p.initpop.data(), n * kGenotypeStride * 4, cudaMemcpyHostToDevice, E.stream);
	if (e == cudaSuccess) e = cudaMemcpyAsync(B + o_pr, p.prng.data(), n * 64 * 4, cudaMemcpyHostToDevice, E.stream);
	if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
	if (e != cudaSuccess) { cudaFree(r->state); r->state = nullptr; return cuda_fail(e, "request upload"); }
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
	d.max_evals = rp->max_evals;
	d.max_gens = rp->max_gens ? rp->max_gens : 0xFFFFFFFFu;
	d.lsmet = rp->lsmet;
	d.runs = runs;
	r->id = E.next_id++;
	r->receptor = rp->receptor;
	r->runs = runs;
	r->bytes = need;
	r->natoms = dp.num_of_atoms;
	r->ntors = dp.num_of_genes - 6;
	r->tpp = E.cfg.threads_per_pose ? E.cfg.threads_per_pose : tune_tpp(E, *r);
	r->t_submit = now_s();
	E.used += need;
	E.stats.submitted++;
	*request_id = r->id;
	E.requests[r->id] = std::move(r);
	return ADGPU_OK;
}

adgpu_status adgpu_engine_tick(adgpu_engine* en, int* completed)
{
	if (!en) return fail(ADGPU_ERR_ARG, "null engine");
	Engine& E = en->e;
	std::lock_guard<std::mutex> lk(E.mu);
	// active requests and their runs, grouped by threads-per-pose class
	std::vector<ReqDev> reqs;
	std::vector<Request*> order;
	constexpr int NC = 12;                 // classes: threads per pose (3) x local search (4)
	std::vector<RunRef> work[NC];
	int max_atoms[NC], max_tors[NC];
	for (int c = 0; c < NC; c++) { max_atoms[c] = 1; max_tors[c] = 0; }
	for (auto& kv : E.requests) {
		Request& r = *kv.second;
		if (r.done) continue;
		int cls = (r.tpp == 32 ? 0 : (r.tpp == 64 ? 1 : 2)) * 4 + r.dev.lsmet;
		int idx = (int)reqs.size();
		reqs.push_back(r.dev);
		order.push_back(&r);
		for (int k = 0; k < r.runs; k++) work[cls].push_back({idx, k});
		max_atoms[cls] = std::max(max_atoms[cls], r.natoms);
		max_tors[cls] = std::max(max_tors[cls], r.ntors);
	}
	if (completed) *completed = 0;
	if (reqs.empty()) return ADGPU_OK;
	size_t nwork = 0;
	for (int c = 0; c < NC; c++) nwork += work[c].size();
	cudaError_t e;
	if ((int)reqs.size() > E.d_reqs_cap) {
		if (E.d_reqs) cudaFree(E.d_reqs);
		E.d_reqs_cap = std::max<int>((int)reqs.size() * 2, 64);
		e = cudaMalloc(&E.d_reqs, sizeof(ReqDev) * E.d_reqs_cap);
		if (e != cudaSuccess) return cuda_fail(e, "request table");
	}
	if ((int)nwork > E.d_work_cap) {
		if (E.d_work) cudaFree(E.d_work);
		E.d_work_cap = std::max<int>((int)nwork * 2, 256);
		e = cudaMalloc(&E.d_work, (sizeof(RunRef) + 1) * E.d_work_cap);
		if (e != cudaSuccess) return cuda_fail(e, "work list");
	}
	std::vector<RunRef> all;
	all.reserve(nwork);
	size_t start[NC];
	for (int c = 0; c < NC; c++) { start[c] = all.size(); all.insert(all.end(), work[c].begin(), work[c].end()); }
	uint8_t* d_done = reinterpret_cast<uint8_t*>(E.d_work + E.d_work_cap);
	e = cudaMemcpyAsync(E.d_reqs, reqs.data(), sizeof(ReqDev) * reqs.size(), cudaMemcpyHostToDevice, E.stream);
	if (e == cudaSuccess) e = cudaMemcpyAsync(E.d_work, all.data(), sizeof(RunRef) * nwork, cudaMemcpyHostToDevice, E.stream);
	if (e == cudaSuccess) e = cudaMemsetAsync(E.d_counters, 0, NC * sizeof(unsigned int), E.stream);
	if (e != cudaSuccess) return cuda_fail(e, "tick upload");
	const int gens = E.cfg.gens_per_tick;
	for (int c = 0; c < NC; c++) {
		if (work[c].empty()) continue;
		adgpu_status st = ADGPU_OK;
		const RunRef* w = E.d_work + start[c];
		uint8_t* wd = d_done + start[c];
		int n = (int)work[c].size();
		unsigned int* ctr = E.d_counters + c;
#define ADGPU_ENGINE_CASE(ID, TPP, LS) \
		case ID: st = launch_engine<TPP, LS>(E, w, wd, n, gens, max_atoms[c], max_tors[c], ctr); break;
		switch (c) {
			ADGPU_ENGINE_CASE(0, 32, LS_SW) ADGPU_ENGINE_CASE(1, 32, LS_AD) ADGPU_ENGINE_CASE(2, 32, LS_ADAM) ADGPU_ENGINE_CASE(3, 32, LS_FIRE)
			ADGPU_ENGINE_CASE(4, 64, LS_SW) ADGPU_ENGINE_CASE(5, 64, LS_AD) ADGPU_ENGINE_CASE(6, 64, LS_ADAM) ADGPU_ENGINE_CASE(7, 64, LS_FIRE)
			ADGPU_ENGINE_CASE(8, 128, LS_SW) ADGPU_ENGINE_CASE(9, 128, LS_AD) ADGPU_ENGINE_CASE(10, 128, LS_ADAM) ADGPU_ENGINE_CASE(11, 128, LS_FIRE)
		}
#undef ADGPU_ENGINE_CASE
		if (st != ADGPU_OK) return st;
	}
	E.h_done.resize(nwork);
	e = cudaMemcpyAsync(E.h_done.data(), d_done, nwork, cudaMemcpyDeviceToHost, E.stream);
	if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
	if (e != cudaSuccess) return cuda_fail(e, "engine tick");
	E.stats.ticks++;
	// a request is complete when all its runs are
	std::vector<int> runs_done(order.size(), 0);
	for (size_t i = 0; i < nwork; i++)
		if (E.h_done[i]) runs_done[all[i].req]++;
	int comp = 0;
	double t = now_s();
	for (size_t i = 0; i < order.size(); i++)
		if (runs_done[i] == order[i]->runs) {
			order[i]->done = true;
			order[i]->t_done = t;
			comp++;
		}
	E.stats.completed += comp;
	if (completed) *completed = comp;
	return ADGPU_OK;
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
	if (r.state) cudaFree(r.state);
	r.state = nullptr;
	E.used -= r.bytes;
	E.requests.erase(it);
	return ADGPU_OK;
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

// Scores a fixed set of poses of the request's ligand with each group size and
// keeps the fastest; cached per (atoms/16, pairs/256) bucket.
template <int TPP>
__global__ void __launch_bounds__(128) tune_kernel(KArgs a, float* grads)
{
	int gid, ngroups;
	Group<TPP> G;
	GroupSmem S;
	group_of<TPP>(a, gid, ngroups, G, S);
	for (uint32_t b = gid; b < a.nblocks; b += ngroups) score_block<TPP, true>(a, b, G, S, grads);
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
	int grid = std::min<int>((int)((a.nblocks + gpc - 1) / gpc), per_sm * sms);
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
