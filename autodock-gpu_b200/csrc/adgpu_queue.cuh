// adgpu_queue.cuh -- the device task ring of the batch/serving engine's
// persistent kernel, and the globaltimer read the persistent kernels share.
//
// A ring of 64-bit slots: a producer reserves positions with one atomicAdd on
// `tail` and writes each slot as (lap << 32) | task word, lap = position / cap
// + 1; a consumer claims a position with a CAS on `head` and waits (bounded)
// for the slot to carry the lap it expects.  Every wait is bounded: a slot
// that is never written sets ctl->err, an empty queue makes an idle worker
// give up after idle_ns, and the whole pop gives up after a fixed number of
// polls.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace adgpu {

struct QueueCtl {
	unsigned long long head;    // next position to pop
	unsigned long long tail;    // next position to push
	int alive;                  // runs not yet retired
	int err;                    // 1: a reserved slot was never written; 2: a pop polled too long
	int workers;                // pose groups that served this ring
	int pad;
	// accounting (globaltimer ns): time pose groups spent on tasks, tasks done,
	// first worker start and last worker exit
	unsigned long long busy_ns, tasks, t_first, t_last;
};

struct TaskRing {
	unsigned long long* slots;  // cap slots
	QueueCtl* ctl;
	uint32_t cap;
	int slot_spin;              // polls of a reserved slot before giving up (err 1)
	long long idle_ns;          // an idle worker stops after this long with the ring empty
};

__device__ __forceinline__ long long global_ns()
{
	long long t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// Next task word, or -1 when the worker should stop: every run has retired,
// `deadline` (globaltimer ns, 0: none) has passed, the ring stayed empty for
// idle_ns, or (error, ctl->err set) a reserved slot was never written.
__device__ inline int ring_pop(const TaskRing& C, long long deadline)
{
	volatile QueueCtl* vq = C.ctl;
	long long idle_since = -1;
	for (int spins = 0; spins < (1 << 28); spins++) {
		if (deadline && global_ns() > deadline) return -1;
		const unsigned long long h = vq->head, t = vq->tail;
		if (h < t) {
			if (atomicCAS(&C.ctl->head, h, h + 1) != h) continue;
			const unsigned long long want = h / C.cap + 1;
			volatile unsigned long long* s = C.slots + (h % C.cap);
			for (int k = 0; k < C.slot_spin; k++) {
				const unsigned long long v = *s;
				if ((v >> 32) == want) {
					__threadfence();
					return (int)(uint32_t)v;
				}
				__nanosleep(64);
			}
			atomicExch(&C.ctl->err, 1);
			return -1;
		}
		if (vq->alive <= 0) return -1;
		const long long now = global_ns();
		if (idle_since < 0) idle_since = now;
		else if (now - idle_since > C.idle_ns) return -1;
		__nanosleep(400);
	}
	atomicExch(&C.ctl->err, 2);
	return -1;
}

// Pushes task words word0 | i, i in [0, n), with a whole pose group; `pos` is
// a shared-memory word of the group.
template <class Group>
__device__ inline void ring_push(const TaskRing& C, uint32_t word0, int n, const Group& G, unsigned long long& pos)
{
	if (G.rank == 0) pos = atomicAdd(&C.ctl->tail, (unsigned long long)n);
	G.sync();
	const unsigned long long p0 = pos;
	__threadfence();
	for (int i = G.rank; i < n; i += G.size()) {
		const unsigned long long p = p0 + (unsigned long long)i;
		atomicExch(C.slots + (p % C.cap), ((p / C.cap + 1) << 32) | (word0 | (uint32_t)i));
	}
	G.sync();
}

}  // namespace adgpu
