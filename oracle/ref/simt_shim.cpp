/*
 * simt_shim.cpp -- cooperative-fiber SIMT emulator behind simt_shim.h.
 * TEST INFRASTRUCTURE ONLY (oracle side).  See simt_shim.h for the model.
 */
#include "simt_shim.h"
#include <ucontext.h>
#include <vector>
#include <thread>
#include <atomic>

thread_local uint3_ adgpu_sim_threadIdx;
thread_local uint3_ adgpu_sim_blockIdx;
thread_local uint3_ adgpu_sim_blockDim;

namespace {

enum FiberState { F_RUNNABLE, F_BLOCK_BAR, F_WARP_BAR, F_DONE };

struct Fiber {
	ucontext_t ctx;
	std::vector<char> stack;
	FiberState state;
	unsigned tid;
};

struct Block {
	ucontext_t sched;
	std::vector<Fiber> fibers;
	unsigned nthreads = 0;
	unsigned cur = 0;
	const std::function<void()>* body = nullptr;
	// block barrier
	unsigned bar_arrived = 0;
	// warp exchange slots
	uint32_t slots[32][32];
	unsigned warp_arrived[32];
};

thread_local Block* g_blk = nullptr;

constexpr size_t kStack = 256 * 1024;

unsigned live_in_block(Block* b) {
	unsigned n = 0;
	for (auto& f : b->fibers) n += (f.state != F_DONE);
	return n;
}

unsigned live_in_warp(Block* b, unsigned w) {
	unsigned n = 0;
	unsigned lo = w * 32, hi = std::min(b->nthreads, lo + 32);
	for (unsigned t = lo; t < hi; t++) n += (b->fibers[t].state != F_DONE);
	return n;
}

void fiber_entry() {
	Block* b = g_blk;
	(*b->body)();
	b->fibers[b->cur].state = F_DONE;
	// a finished fiber may complete a pending block barrier
	if (b->bar_arrived > 0 && b->bar_arrived == live_in_block(b)) {
		b->bar_arrived = 0;
		for (auto& f : b->fibers) if (f.state == F_BLOCK_BAR) f.state = F_RUNNABLE;
	}
	swapcontext(&b->fibers[b->cur].ctx, &b->sched);
}

void park(Block* b) {
	swapcontext(&b->fibers[b->cur].ctx, &b->sched);
	adgpu_sim_threadIdx.x = b->cur;
}

void warp_wait(Block* b) {
	unsigned w = b->cur / 32;
	b->warp_arrived[w]++;
	if (b->warp_arrived[w] == live_in_warp(b, w)) {
		b->warp_arrived[w] = 0;
		unsigned lo = w * 32, hi = std::min(b->nthreads, lo + 32);
		for (unsigned t = lo; t < hi; t++)
			if (b->fibers[t].state == F_WARP_BAR) b->fibers[t].state = F_RUNNABLE;
		return;  // last arriver continues without parking
	}
	b->fibers[b->cur].state = F_WARP_BAR;
	park(b);
}

void run_block(unsigned bid, unsigned nthreads, const std::function<void()>& body) {
	static thread_local Block blk;
	blk.nthreads = nthreads;
	blk.cur = 0;
	blk.bar_arrived = 0;
	blk.body = &body;
	memset(blk.warp_arrived, 0, sizeof(blk.warp_arrived));
	blk.fibers.resize(nthreads);
	Block* saved = g_blk;
	g_blk = &blk;
	adgpu_sim_blockIdx.x = bid; adgpu_sim_blockIdx.y = 0; adgpu_sim_blockIdx.z = 0;
	adgpu_sim_blockDim.x = nthreads; adgpu_sim_blockDim.y = 1; adgpu_sim_blockDim.z = 1;
	for (unsigned t = 0; t < nthreads; t++) {
		Fiber& f = blk.fibers[t];
		if (f.stack.size() != kStack) f.stack.resize(kStack);
		f.state = F_RUNNABLE;
		f.tid = t;
		getcontext(&f.ctx);
		f.ctx.uc_stack.ss_sp = f.stack.data();
		f.ctx.uc_stack.ss_size = kStack;
		f.ctx.uc_link = nullptr;
		makecontext(&f.ctx, (void (*)())fiber_entry, 0);
	}
	for (;;) {
		bool progressed = false, all_done = true;
		for (unsigned t = 0; t < nthreads; t++) {
			Fiber& f = blk.fibers[t];
			if (f.state != F_DONE) all_done = false;
			if (f.state != F_RUNNABLE) continue;
			blk.cur = t;
			adgpu_sim_threadIdx.x = t; adgpu_sim_threadIdx.y = 0; adgpu_sim_threadIdx.z = 0;
			swapcontext(&blk.sched, &f.ctx);
			progressed = true;
		}
		if (all_done) break;
		if (!progressed) {
			fprintf(stderr, "simt_shim: deadlock in block %u\n", bid);
			abort();
		}
	}
	g_blk = saved;
}

}  // namespace

void adgpu_sim_syncthreads() {
	Block* b = g_blk;
	b->bar_arrived++;
	if (b->bar_arrived == live_in_block(b)) {
		b->bar_arrived = 0;
		for (auto& f : b->fibers) if (f.state == F_BLOCK_BAR) f.state = F_RUNNABLE;
		return;
	}
	b->fibers[b->cur].state = F_BLOCK_BAR;
	park(b);
}

uint32_t adgpu_sim_shfl_bits(uint32_t bits, int src_lane) {
	Block* b = g_blk;
	unsigned w = b->cur / 32, lane = b->cur % 32;
	b->slots[w][lane] = bits;
	warp_wait(b);
	uint32_t r = b->slots[w][((unsigned)src_lane) % 32];
	warp_wait(b);
	return r;
}

int adgpu_sim_any(int pred) {
	Block* b = g_blk;
	unsigned w = b->cur / 32, lane = b->cur % 32;
	b->slots[w][lane] = pred ? 1u : 0u;
	warp_wait(b);
	unsigned lo = w * 32, hi = std::min(b->nthreads, lo + 32);
	int any = 0;
	for (unsigned t = lo; t < hi; t++)
		if (b->fibers[t].state != F_DONE && b->slots[w][t - lo]) any = 1;
	warp_wait(b);
	return any;
}

void adgpu_ref_launch(unsigned blocks, unsigned threads, const std::function<void()>& body) {
	unsigned nworkers = 1;
	if (const char* e = getenv("ADGPU_REF_THREADS")) nworkers = (unsigned)atoi(e);
	if (nworkers < 1) nworkers = 1;
	if (nworkers > blocks) nworkers = blocks ? blocks : 1;
	if (nworkers == 1) {
		for (unsigned b = 0; b < blocks; b++) run_block(b, threads, body);
		return;
	}
	std::atomic<unsigned> next(0);
	std::vector<std::thread> pool;
	for (unsigned w = 0; w < nworkers; w++)
		pool.emplace_back([&]() {
			for (;;) {
				unsigned b = next.fetch_add(1);
				if (b >= blocks) break;
				run_block(b, threads, body);
			}
		});
	for (auto& t : pool) t.join();
}
