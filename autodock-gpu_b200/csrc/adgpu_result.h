// adgpu_result.h -- result processing core shared by the kernel-API entry
// (adgpu_process_result) and the engine (adgpu_engine_process_result).
#pragma once
#include <cuda_runtime.h>
#include "adgpu_prep.h"

namespace adgpu {

// grid: device maps, grid_cells 0 for the reference layout (4 floats per
// point per map), 1 for the engine's 8-corner cell records.  populations and
// energies are device buffers, ordered in place; scratch comes from `pool`
// when given (else the device's default pool), on stream `st`, which is
// synchronised before returning.
adgpu_status process_result_core(const PostLigand& L, const uint32_t* pairs, const adgpu_dockpars& dp,
                                 const float* grid, int grid_cells, float* populations, float* energies,
                                 uint32_t num_runs, const adgpu_result_params* params, adgpu_run_result* runs_out,
                                 adgpu_cluster* clusters_out, int* num_clusters, double* best_xyz, float* peratom,
                                 float* entities, cudaStream_t st, cudaMemPool_t pool);

}  // namespace adgpu
