// adgpu_api.cu -- kernels, table repacking and the C ABI of the reference
// kernel API (include/adgpu_b200.h, layer 1).
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <mutex>

#include "adgpu_kernels.cuh"
#include "adgpu_autostop.cuh"
#include "adgpu_tables.h"
#include "adgpu_pipeline.h"
#include "adgpu_nvtx.h"

#ifndef ADGPU_MIN_CTAS
#define ADGPU_MIN_CTAS 6     // 6 CTAs x 4 warps per SM: <= 80 registers, no spills
#endif
// The gradient local searches (ADADELTA, ADAM, FIRE) need more registers than
// 80 for their scorer without spills; the SM's throughput is the same with 5
// CTAs as with 6 (the scorer is issue bound).
#ifndef ADGPU_MIN_CTAS_GRAD
#define ADGPU_MIN_CTAS_GRAD 5
#endif

namespace adgpu {

thread_local std::string g_last_error;

adgpu_status fail(adgpu_status st, const std::string& msg)
{
	g_last_error = msg;
	return st;
}

adgpu_status cuda_fail(cudaError_t e, const char* what)
{
	g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
	return ADGPU_ERR_CUDA;
}

#define ADGPU_CUDA(call, what) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return cuda_fail(e_, what); } while (0)

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
constexpr int lga_min_ctas(int kind) { return kind >= 2 && kind <= 4 ? ADGPU_MIN_CTAS_GRAD : ADGPU_MIN_CTAS; }

template <int TPP, int KIND>
__global__ void __launch_bounds__(128, lga_min_ctas(KIND)) lga_kernel(KArgs a, float* grads)
{
	if (a.stop_flag && *a.stop_flag) return;
	int gid, ngroups;
	Group<TPP> G;
	GroupSmem S;
	group_of<TPP>(a, gid, ngroups, G, S);
	// Local searches run for a data-dependent number of iterations, so pose
	// groups take the next block from a counter instead of a fixed stride.
	auto next = [&](uint32_t cur) -> uint32_t {
		if (a.work_counter == nullptr) return cur + ngroups;
		uint32_t b = 0;
		if (G.rank == 0) b = atomicAdd(a.work_counter, 1u) + (uint32_t)ngroups;
		if constexpr (TPP == 32) {
			b = __shfl_sync(0xffffffffu, b, 0);
		} else {
			if (G.rank == 0) S.misc[15] = (int)b;
			G.sync();
			b = (uint32_t)S.misc[15];
			G.sync();
		}
		return b;
	};
	for (uint32_t b = gid; b < a.nblocks; b = next(b)) {
		if constexpr (KIND == 0) ga_block<TPP>(a, b, G, S);
		else if constexpr (KIND == 1) sw_block<TPP>(a, b, G, S);
		else if constexpr (KIND == 2) gradient_ls_block<TPP, LS_AD>(a, b, G, S);
		else if constexpr (KIND == 3) gradient_ls_block<TPP, LS_ADAM>(a, b, G, S);
		else if constexpr (KIND == 4) fire_block<TPP>(a, b, G, S);
		else if constexpr (KIND == 5) initpop_block<TPP>(a, b, G, S);
		else if constexpr (KIND == 6) score_block<TPP, false>(a, b, G, S, grads);
		else if constexpr (KIND == 7) score_block<TPP, true>(a, b, G, S, grads);
		else if constexpr (KIND == 8) score_terms_block<TPP>(a, b, G, S, grads);
	}
}

// Per-run eval sums (cuda/kernel2.cu:26-52): one warp per run.
__global__ void sum_evals_kernel(const int* evals_new, int* evals_runs, int pop_size, int runs, const int* stop_flag)
{
	if (stop_flag && *stop_flag) return;
	int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
	if (w >= runs) return;
	int s = 0;
	for (int i = lane; i < pop_size; i += 32) s += evals_new[w * pop_size + i];
	for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
	if (lane == 0) evals_runs[w] += s;
}

// Stop test of the resident docking loop (check_progress,
// host/src/performdocking.cpp.Cuda:908-942): stop when the mean evals per run
// reach max_evals or the generation count reaches max_gens.
// With AutoStop (as != nullptr), a generation count that is a multiple of
// as_frequency also runs the AutoStop check on the current energies and stops
// once it is satisfied and the evaluations exceed min_as_evals
// (performdocking.cpp.Cuda:689-698).  Launch with 256 threads.
struct AutoStopArgs {
	AutoStopState* state;        // nullptr: no AutoStop
	float* stats;                // (pop_size + 1) * 3
	float* buf_e;                // R * P
	uint16_t* buf_m;             // R * P
	const float* energies;       // the population about to be bred
	unsigned long long min_evals;
};

__global__ void __launch_bounds__(256) progress_kernel(const int* evals_runs, int runs, unsigned long long max_evals,
                                                       unsigned int max_gens, unsigned int* gen_counter, int* stop_flag,
                                                       AutoStopArgs as)
{
	if (*stop_flag) return;
	__shared__ unsigned long long tot;
	__shared__ int s_stop;
	__shared__ int s_count[257];
	__shared__ float s_best[256];
	if (threadIdx.x == 0) tot = 0;
	__syncthreads();
	unsigned long long s = 0;
	for (int i = threadIdx.x; i < runs; i += blockDim.x) s += (unsigned long long)evals_runs[i];
	atomicAdd(&tot, s);
	__syncthreads();
	const unsigned int g = *gen_counter;
	if (threadIdx.x == 0) {
		double ev = (double)tot / (double)runs / (double)max_evals * 100.0;
		double gp = (double)g / (double)max_gens * 100.0;
		s_stop = (ev > gp ? ev : gp) >= 100.0;
	}
	__syncthreads();
	if (!s_stop && as.state && g % as.state->as_frequency == 0) {
		autostop_check(*as.state, as.stats, as.buf_e, as.buf_m, as.energies, (int)g, s_count, s_best);
		if (threadIdx.x == 0 && as.state->autostopped && tot > as.min_evals) s_stop = 1;
	}
	if (threadIdx.x == 0) {
		if (s_stop) *stop_flag = 1;
		else *gen_counter = g + 1;
	}
}

// Relayout of the reference grid (4 replicated floats per point,
// host/src/processgrid.cpp:244-248) into 32-byte cell records: for cell c and
// map slot s the record holds the same 8 floats the reference reads from
// fgrids + ((map*g3 + p) << 2), p = the cell's lower corner.
__global__ void relayout_grid_kernel(const float* __restrict__ ref, float* __restrict__ out,
                                     int gx, int gy, int gz, int nmaps, int num_map_atypes)
{
	const size_t cx = gx - 1, cy = gy - 1, cz = gz - 1;
	const size_t ncells = cx * cy * cz;
	const size_t g3 = (size_t)gx * gy * gz;
	const size_t total = ncells * nmaps;
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
		size_t cell = i / nmaps;
		int slot = (int)(i - cell * nmaps);
		size_t x = cell % cx, y = (cell / cx) % cy, z = cell / (cx * cy);
		int map = slot == 0 ? num_map_atypes : (slot == 1 ? num_map_atypes + 1 : slot - 2);
		size_t p = x + y * gx + z * (size_t)gx * gy;
		const float4* src = reinterpret_cast<const float4*>(ref + (((size_t)map * g3 + p) << 2));
		float4* dst = reinterpret_cast<float4*>(out + i * 8);
		dst[0] = src[0];
		dst[1] = src[1];
	}
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
int g_num_sms = 0;

template <int TPP, int KIND>
adgpu_status launch_lga(const KArgs& a, float* grads, cudaStream_t stream, int cta_threads)
{
	if (a.nblocks == 0) return ADGPU_OK;
	const int gpc = cta_threads / TPP;
	const int bytes = group_smem_bytes(a.L.natoms, a.L.ntors, (int)a.ref_threads, TPP) * gpc;
	auto kfn = lga_kernel<TPP, KIND>;
	if (bytes > 48 * 1024) ADGPU_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes), "smem attribute");
	static int carveout = -2;           // per instantiation: the last preference set
	const int pct = smem_carveout_pct(bytes, lga_min_ctas(KIND));
	if (pct >= 0 && pct > carveout) {
		ADGPU_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributePreferredSharedMemoryCarveout, pct), "carveout");
		carveout = pct;
	}
	int per_sm = 0;
	ADGPU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, cta_threads, bytes), "occupancy");
	if (per_sm < 1) return fail(ADGPU_ERR_LIMIT, "kernel does not fit on an SM");
	if (g_num_sms == 0) {
		int dev; ADGPU_CUDA(cudaGetDevice(&dev), "device");
		ADGPU_CUDA(cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev), "sm count");
	}
	long need = ((long)a.nblocks + gpc - 1) / gpc;
	long cap = (long)per_sm * g_num_sms;
	int grid = (int)(need < cap ? need : cap);
	kfn<<<grid, cta_threads, bytes, stream>>>(a, grads);
	ADGPU_CUDA(cudaGetLastError(), "kernel launch");
	return ADGPU_OK;
}

// Threads per pose for a launch of n blocks when none is configured.
// Solis-Wets and ADADELTA: 64.  Their searches stop on their own step-size
// test, so a launch ends with its longest entities running alone, and two
// warps per pose halve that tail; on B200, 64 beat 32 and 128 for per-ligand
// dockings of 20 and of 100 runs (80% local-search rate, 10-64 heavy atoms;
// 100 runs of 40 heavy atoms: ADADELTA 121 vs 116 M evals/s, Solis-Wets 242
// vs 232).  ADAM and FIRE run a fixed number of iterations, so there is no
// tail to shorten and throughput decides: 32 (ADAM 163 vs 146, FIRE 138 vs
// 119 M evals/s at 100 runs) unless the launch leaves pose groups idle.
// Other kernels: 64 when every block still gets a resident pose group of 64
// threads (6 CTAs of 128 threads per SM), else 32.
static int auto_tpp(uint32_t n, int kind)
{
	if (kind == 1 || kind == 2) return 64;
	if (g_num_sms == 0) {
		int dev = 0;
		if (cudaGetDevice(&dev) != cudaSuccess ||
		    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 32;
	}
	const long groups32 = (long)g_num_sms * ADGPU_MIN_CTAS * 4;
	return (long)n * 2 <= groups32 ? 64 : 32;
}

template <int KIND>
adgpu_status launch_kind(const KArgs& a, float* grads, cudaStream_t stream, int tpp)
{
	if (tpp == 0) tpp = auto_tpp(a.nblocks, KIND);
	switch (tpp) {
	case 32: return launch_lga<32, KIND>(a, grads, stream, 128);
	case 64: return launch_lga<64, KIND>(a, grads, stream, 128);
	case 128: return launch_lga<128, KIND>(a, grads, stream, 128);
	default: return fail(ADGPU_ERR_ARG, "threads per pose must be 32, 64 or 128");
	}
}

// ---------------------------------------------------------------------------
// state of the reference-API path (one ligand at a time, like the reference's
// single __constant__ GpuData, cuda/kernels.cu:123)
// ---------------------------------------------------------------------------
struct ApiState {
	bool ready = false;
	adgpu_gpudata data;
	LigandTables tables;       // host-repacked + device copy
	int tpp = 0;               // threads per pose; 0: chosen per launch (auto_tpp)
	unsigned int* counters = nullptr;   // library-owned work counters of the local-search launches
	bool pipeline = true;      // adgpu_dock_resident without AutoStop runs the pipelined loop where it applies
	PipeScratch pipe;          // its scratch, kept between calls
	std::mutex mu;
};

ApiState& api()
{
	static ApiState s;
	return s;
}

KArgs make_args(ApiState& s)
{
	KArgs a;
	memset(&a, 0, sizeof(a));
	a.L = s.tables.dev;
	a.dp = s.data.dockpars;
	a.prng = s.data.pMem_prng_states;
	a.evals_new = s.data.pMem_evals_of_new_entities;
	a.evals_runs = s.data.pMem_gpu_evals_of_runs;
	a.ref_threads = 64;
	return a;
}

adgpu_status check_threads(uint32_t threads)
{
	if (threads == 0 || threads > 256) return fail(ADGPU_ERR_ARG, "threads must be 1..256");
	return ADGPU_OK;
}


// Resident docking loop: the generation loop of docking_with_gpu
// (host/src/performdocking.cpp.Cuda:684-831) with the stop test on the device
// and two generations (A->B, B->A) captured in one CUDA graph, so the host
// only launches graphs and polls a pinned stop flag every few generations.
adgpu_status dock_resident(ApiState& s, int lsmet, uint32_t runs, uint64_t max_evals, uint32_t max_gens,
                           uint32_t as_frequency, float stopstd, uint64_t min_as_evals,
                           float* c1, float* e1, float* c2, float* e2, int* final_is_second, uint32_t* generations,
                           int* autostopped)
{
	const adgpu_dockpars& dp = s.data.dockpars;
	memset(&s.pipe.stats, 0, sizeof(s.pipe.stats));
	if (as_frequency == 0 && s.pipeline && pipeline_applies(dp, runs)) {
		*autostopped = 0;
		KArgs base = make_args(s);
		return dock_pipelined(base, s.pipe, lsmet, s.tpp, runs, max_evals, max_gens, c1, e1, c2, e2,
		                      final_is_second, generations);
	}
	const uint32_t T = 64;
	cudaStream_t st;
	ADGPU_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
	int* d_flag = nullptr; unsigned int* d_gen = nullptr;
	int* h_flag = nullptr;
	char* d_as = nullptr;                // AutoStop state, statistics and buffers
	cudaGraph_t graph = nullptr; cudaGraphExec_t exec = nullptr;
	adgpu_status rc = ADGPU_OK;
	auto cleanup = [&]() {
		if (exec) cudaGraphExecDestroy(exec);
		if (graph) cudaGraphDestroy(graph);
		if (d_flag) cudaFree(d_flag);
		if (d_gen) cudaFree(d_gen);
		if (d_as) cudaFree(d_as);
		if (h_flag) cudaFreeHost(h_flag);
		cudaStreamDestroy(st);
	};
#define ADGPU_TRY(call, what) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { rc = cuda_fail(e_, what); cleanup(); return rc; } } while (0)
	ADGPU_TRY(cudaMalloc(&d_flag, sizeof(int)), "flag");
	ADGPU_TRY(cudaMalloc(&d_gen, sizeof(unsigned int)), "gen counter");
	ADGPU_TRY(cudaMallocHost(&h_flag, 8 * sizeof(int)), "pinned flags");
	ADGPU_TRY(cudaMemsetAsync(d_flag, 0, sizeof(int), st), "flag init");
	ADGPU_TRY(cudaMemsetAsync(d_gen, 0, sizeof(unsigned int), st), "gen init");
	AutoStopArgs as_args{};
	if (as_frequency > 0) {
		const size_t n = (size_t)runs * dp.pop_size;
		const size_t o_stats = 256, o_e = o_stats + autostop_stats_floats(dp.pop_size) * 4;
		const size_t o_m = (o_e + n * 4 + 15) / 16 * 16, bytes = o_m + n * 2 + 16;
		ADGPU_TRY(cudaMalloc(&d_as, bytes), "autostop state");
		AutoStopState h;
		autostop_init(h, dp.pop_size, (int)runs, stopstd, as_frequency);
		ADGPU_TRY(cudaMemcpyAsync(d_as, &h, sizeof(h), cudaMemcpyHostToDevice, st), "autostop init");
		as_args.state = reinterpret_cast<AutoStopState*>(d_as);
		as_args.stats = reinterpret_cast<float*>(d_as + o_stats);
		as_args.buf_e = reinterpret_cast<float*>(d_as + o_e);
		as_args.buf_m = reinterpret_cast<uint16_t*>(d_as + o_m);
		as_args.min_evals = min_as_evals;
	}
	KArgs a = make_args(s);
	a.ref_threads = T;
	a.stop_flag = d_flag;
	const int ls_kind = lsmet == 0 ? 1 : (lsmet == 1 ? 2 : (lsmet == 2 ? 3 : 4));
	ADGPU_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
	for (int half = 0; half < 2; half++) {
		float* cc = half ? c2 : c1; float* ec = half ? e2 : e1;
		float* cn = half ? c1 : c2; float* en = half ? e1 : e2;
		AutoStopArgs ash = as_args;
		ash.energies = ec;
		progress_kernel<<<1, 256, 0, st>>>(s.data.pMem_gpu_evals_of_runs, (int)runs, (unsigned long long)max_evals, max_gens,
		                                   d_gen, d_flag, ash);
		KArgs g = a;
		g.nblocks = runs * (uint32_t)dp.pop_size;
		g.conf_cur = cc; g.e_cur = ec; g.conf = cn; g.e = en;
		rc = launch_kind<0>(g, nullptr, st, s.tpp);
		if (rc == ADGPU_OK && dp.lsearch_rate != 0.0f) {
			KArgs l = a;
			l.nblocks = runs * dp.num_of_lsentities;
			l.conf = cn; l.e = en;
			l.work_counter = s.counters + 1 + half;
			cudaMemsetAsync(l.work_counter, 0, sizeof(unsigned int), st);
			switch (ls_kind) {
			case 1: rc = launch_kind<1>(l, nullptr, st, s.tpp); break;
			case 2: rc = launch_kind<2>(l, nullptr, st, s.tpp); break;
			case 3: rc = launch_kind<3>(l, nullptr, st, s.tpp); break;
			default: rc = launch_kind<4>(l, nullptr, st, s.tpp); break;
			}
		}
		if (rc != ADGPU_OK) { cudaStreamEndCapture(st, &graph); cleanup(); return rc; }
		sum_evals_kernel<<<(runs + 3) / 4, 128, 0, st>>>(s.data.pMem_evals_of_new_entities, s.data.pMem_gpu_evals_of_runs,
		                                                dp.pop_size, (int)runs, d_flag);
	}
	ADGPU_TRY(cudaStreamEndCapture(st, &graph), "end capture");
	ADGPU_TRY(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
	// Graphs go out in batches of kPoll, each followed by a copy of the stop
	// flag and an event.  The host keeps kAhead batches queued behind the one
	// whose flag it waits for (48 generations, about 0.4 s of work at the
	// plain workload), so a host thread that is descheduled for a while does
	// not leave the GPU idle (with one batch queued, 8 of 27 plain dockings
	// took 10-30 % longer on a shared host; with three, 2 of 27).  Once the
	// flag is set every kernel returns at entry, so the batches queued past
	// the stop cost only their launches (under 1 ms).
	const int kPoll = 4;     // graphs (2 generations each) per batch
	const int kAhead = 6;    // batches queued beyond the one being waited for
	const int kSlots = kAhead + 1;
	cudaEvent_t ev[kSlots] = {};
	auto cleanup_ev = [&]() { for (auto& x : ev) if (x) { cudaEventDestroy(x); x = nullptr; } };
	for (auto& x : ev)
		if (cudaEventCreateWithFlags(&x, cudaEventDisableTiming) != cudaSuccess) { cleanup_ev(); cleanup(); return fail(ADGPU_ERR_CUDA, "events"); }
	auto queue_batch = [&](int slot) -> cudaError_t {
		for (int i = 0; i < kPoll; i++) {
			cudaError_t e = cudaGraphLaunch(exec, st);
			if (e != cudaSuccess) return e;
		}
		cudaError_t e = cudaMemcpyAsync(h_flag + slot, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st);
		return e == cudaSuccess ? cudaEventRecord(ev[slot], st) : e;
	};
	cudaError_t qe = cudaSuccess;
	for (int k = 0; k < kAhead && qe == cudaSuccess; k++) qe = queue_batch(k);
	for (int k = 0; qe == cudaSuccess; k++) {
		qe = queue_batch((k + kAhead) % kSlots);
		if (qe == cudaSuccess) qe = cudaEventSynchronize(ev[k % kSlots]);
		if (qe == cudaSuccess && h_flag[k % kSlots]) break;
	}
	if (qe == cudaSuccess) qe = cudaStreamSynchronize(st);
	cleanup_ev();
	ADGPU_TRY(qe, "generation loop");
	unsigned int g = 0;
	ADGPU_TRY(cudaMemcpy(&g, d_gen, sizeof(g), cudaMemcpyDeviceToHost), "gen read");
	*generations = g;
	*final_is_second = (int)(g & 1u);
	s.pipe.stats.generations = g;
	*autostopped = 0;
	if (as_args.state) {
		AutoStopState h;
		ADGPU_TRY(cudaMemcpy(&h, as_args.state, sizeof(h), cudaMemcpyDeviceToHost), "autostop read");
		*autostopped = h.autostopped;
	}
	cleanup();
#undef ADGPU_TRY
	return ADGPU_OK;
}

}  // namespace adgpu

using namespace adgpu;

extern "C" {

const char* adgpu_last_error(void) { return g_last_error.c_str(); }
const char* adgpu_version(void) { return "adgpu_b200 0.1 (sm_100a)"; }

adgpu_status adgpu_set_kernels_gpu_data(const adgpu_gpudata* data)
{
	if (!data) return fail(ADGPU_ERR_ARG, "null GpuData");
	ApiState& s = api();
	std::lock_guard<std::mutex> lk(s.mu);
	s.ready = false;
	s.data = *data;
	adgpu_status st = build_ligand_tables_from_device(*data, s.tables);
	if (st != ADGPU_OK) return st;
	s.tpp = 0;
	if (const char* t = getenv("ADGPU_THREADS_PER_POSE")) s.tpp = atoi(t);
	s.pipeline = true;
	if (const char* t = getenv("ADGPU_DOCK_PIPELINE")) s.pipeline = atoi(t) != 0;
	if (!s.counters) ADGPU_CUDA(cudaMalloc(&s.counters, 16 * sizeof(unsigned int)), "work counters");
	s.ready = true;
	return ADGPU_OK;
}

adgpu_status adgpu_get_kernels_gpu_data(adgpu_gpudata* data)
{
	if (!data) return fail(ADGPU_ERR_ARG, "null GpuData");
	ApiState& s = api();
	if (!s.ready) return fail(ADGPU_ERR_NOT_READY, "adgpu_set_kernels_gpu_data not called");
	*data = s.data;
	return ADGPU_OK;
}

static adgpu_status run_kind(int kind, uint32_t blocks, uint32_t threads, const float* cc, const float* ec,
                             float* conf, float* e, float* grads)
{
	ApiState& s = api();
	if (!s.ready) return fail(ADGPU_ERR_NOT_READY, "adgpu_set_kernels_gpu_data not called");
	adgpu_status st = check_threads(threads);
	if (st != ADGPU_OK) return st;
	KArgs a = make_args(s);
	a.ref_threads = threads;
	a.nblocks = blocks;
	a.conf_cur = cc; a.e_cur = ec; a.conf = conf; a.e = e;
	if (kind >= 1 && kind <= 4) {
		ADGPU_CUDA(cudaMemsetAsync(s.counters, 0, sizeof(unsigned int), 0), "work counter reset");
		a.work_counter = s.counters;
	}
	switch (kind) {
	case 0: st = launch_kind<0>(a, grads, 0, s.tpp); break;
	case 1: st = launch_kind<1>(a, grads, 0, s.tpp); break;
	case 2: st = launch_kind<2>(a, grads, 0, s.tpp); break;
	case 3: st = launch_kind<3>(a, grads, 0, s.tpp); break;
	case 4: st = launch_kind<4>(a, grads, 0, s.tpp); break;
	case 5: st = launch_kind<5>(a, grads, 0, s.tpp); break;
	case 6: st = launch_kind<6>(a, grads, 0, s.tpp); break;
	case 7: st = launch_kind<7>(a, grads, 0, s.tpp); break;
	case 8: st = launch_kind<8>(a, grads, 0, s.tpp); break;
	default: return fail(ADGPU_ERR_ARG, "bad kernel kind");
	}
	if (st != ADGPU_OK) return st;
	ADGPU_CUDA(cudaDeviceSynchronize(), "kernel execution");
	return ADGPU_OK;
}

adgpu_status adgpu_calc_initpop(uint32_t blocks, uint32_t threads, float* conf_cur, float* e_cur)
{
	return run_kind(5, blocks, threads, nullptr, nullptr, conf_cur, e_cur, nullptr);
}

adgpu_status adgpu_sum_evals(uint32_t blocks, uint32_t threads)
{
	ApiState& s = api();
	if (!s.ready) return fail(ADGPU_ERR_NOT_READY, "adgpu_set_kernels_gpu_data not called");
	(void)threads;
	int warps_per_cta = 4;
	int grid = (int)((blocks + warps_per_cta - 1) / warps_per_cta);
	if (grid == 0) return ADGPU_OK;
	sum_evals_kernel<<<grid, 32 * warps_per_cta>>>(s.data.pMem_evals_of_new_entities, s.data.pMem_gpu_evals_of_runs,
	                                                s.data.dockpars.pop_size, (int)blocks, nullptr);
	ADGPU_CUDA(cudaGetLastError(), "sum_evals launch");
	ADGPU_CUDA(cudaDeviceSynchronize(), "sum_evals");
	return ADGPU_OK;
}

adgpu_status adgpu_gen_and_eval_newpops(uint32_t blocks, uint32_t threads, float* cc, float* ec, float* cn, float* en)
{
	return run_kind(0, blocks, threads, cc, ec, cn, en, nullptr);
}

adgpu_status adgpu_perform_ls(uint32_t blocks, uint32_t threads, float* cn, float* en)
{
	return run_kind(1, blocks, threads, nullptr, nullptr, cn, en, nullptr);
}

adgpu_status adgpu_gradient_minad(uint32_t blocks, uint32_t threads, float* cn, float* en)
{
	return run_kind(2, blocks, threads, nullptr, nullptr, cn, en, nullptr);
}

adgpu_status adgpu_gradient_minadam(uint32_t blocks, uint32_t threads, float* cn, float* en)
{
	return run_kind(3, blocks, threads, nullptr, nullptr, cn, en, nullptr);
}

adgpu_status adgpu_gradient_minfire(uint32_t blocks, uint32_t threads, float* cn, float* en)
{
	return run_kind(4, blocks, threads, nullptr, nullptr, cn, en, nullptr);
}

adgpu_status adgpu_score_genotypes(uint32_t n, const float* genotypes, float* energies, float* gradients)
{
	return run_kind(gradients ? 7 : 6, n, 64, nullptr, nullptr, const_cast<float*>(genotypes), energies, gradients);
}

adgpu_status adgpu_score_terms(uint32_t n, const float* genotypes, float* energies, float* terms)
{
	if (!genotypes || !energies || !terms) return fail(ADGPU_ERR_ARG, "null buffer");
	return run_kind(8, n, 64, nullptr, nullptr, const_cast<float*>(genotypes), energies, terms);
}

adgpu_status adgpu_dock_stats_get(adgpu_dock_stats* out)
{
	if (!out) return fail(ADGPU_ERR_ARG, "null out");
	*out = api().pipe.stats;
	return ADGPU_OK;
}

adgpu_status adgpu_dock_resident(int lsmet, uint32_t num_runs, uint64_t max_evals, uint32_t max_gens,
                                 float* c1, float* e1, float* c2, float* e2,
                                 int* final_is_second, uint32_t* generations)
{
	adgpu::NvtxRange nvtx_range("adgpu_dock_resident");
	ApiState& s = api();
	if (!s.ready) return fail(ADGPU_ERR_NOT_READY, "adgpu_set_kernels_gpu_data not called");
	if (lsmet < 0 || lsmet > 3) return fail(ADGPU_ERR_ARG, "lsmet must be 0 (sw), 1 (ad), 2 (adam) or 3 (fire)");
	if (!c1 || !e1 || !c2 || !e2 || !final_is_second || !generations) return fail(ADGPU_ERR_ARG, "null buffer");
	if (num_runs == 0 || num_runs > ADGPU_MAX_RUNS || max_evals == 0 || max_gens == 0) return fail(ADGPU_ERR_ARG, "bad run limits");
	int as = 0;
	return dock_resident(s, lsmet, num_runs, max_evals, max_gens, 0, 0.0f, 0, c1, e1, c2, e2, final_is_second, generations, &as);
}

adgpu_status adgpu_dock_resident_autostop(int lsmet, uint32_t num_runs, uint64_t max_evals, uint32_t max_gens,
                                          uint32_t as_frequency, float stopstd, uint64_t min_as_evals,
                                          float* c1, float* e1, float* c2, float* e2,
                                          int* final_is_second, uint32_t* generations, int* autostopped)
{
	adgpu::NvtxRange nvtx_range("adgpu_dock_resident_autostop");
	ApiState& s = api();
	if (!s.ready) return fail(ADGPU_ERR_NOT_READY, "adgpu_set_kernels_gpu_data not called");
	if (lsmet < 0 || lsmet > 3) return fail(ADGPU_ERR_ARG, "lsmet must be 0 (sw), 1 (ad), 2 (adam) or 3 (fire)");
	if (!c1 || !e1 || !c2 || !e2 || !final_is_second || !generations || !autostopped) return fail(ADGPU_ERR_ARG, "null buffer");
	if (num_runs == 0 || num_runs > ADGPU_MAX_RUNS || max_evals == 0 || max_gens == 0) return fail(ADGPU_ERR_ARG, "bad run limits");
	if (as_frequency == 0) return fail(ADGPU_ERR_ARG, "as_frequency must be at least 1");
	if (!(stopstd > 0.0f)) return fail(ADGPU_ERR_ARG, "stopstd must be positive");
	if (s.data.dockpars.pop_size < 11) return fail(ADGPU_ERR_ARG, "AutoStop needs a population of at least 11");
	return dock_resident(s, lsmet, num_runs, max_evals, max_gens, as_frequency, stopstd, min_as_evals,
	                     c1, e1, c2, e2, final_is_second, generations, autostopped);
}

}  // extern "C"
