// adgpu_pipeline.h -- the pipelined plain docking loop (adgpu_pipeline.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include "adgpu_kernels.cuh"
#include "adgpu_tables.h"

#define ADGPU_CUDA_RET(call, what) \
	do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return ::adgpu::cuda_fail(e_, what); } while (0)

namespace adgpu {

// Most population buffers of the pipelined loop (the caller's two plus the
// library's); with nbuf of them runs may run up to nbuf-1 generations ahead
// of the stop test.
constexpr int kPipeBufs = 8;

// Library-owned device scratch of the pipelined loop, kept between calls.
struct PipeScratch {
	void* mem = nullptr;
	size_t bytes = 0;
	long long* host_out = nullptr;   // pinned readback of the loop's outcome
	adgpu_dock_stats stats{};        // accounting of the last call
};

// Whether the pipelined loop can dock these settings with the reference's
// results: every run's local searches must draw only on its own PRNG states,
// which holds when the local-search rate is 100 % (num_of_lsentities ==
// pop_size, host/src/performdocking.cpp.Cuda:446).
bool pipeline_applies(const adgpu_dockpars& dp, uint32_t runs);

// The generation loop of docking_with_gpu as one persistent launch; the
// arguments and results are those of adgpu_dock_resident.  tpp 0: default.
adgpu_status dock_pipelined(const KArgs& base, PipeScratch& sc, int lsmet, int tpp, uint32_t runs,
                            uint64_t max_evals, uint32_t max_gens, float* c1, float* e1, float* c2, float* e2,
                            int* final_is_second, uint32_t* generations);

}  // namespace adgpu
