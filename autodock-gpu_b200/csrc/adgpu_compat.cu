// adgpu_compat.cu -- the reference kernel API under its original C++ names
// and signatures (declared in host/src/performdocking.cpp.Cuda:40-84), so the
// reference host objects (docking_with_gpu and the rest of host/src) link
// against libadgpu_b200 instead of cuda/kernels.o without a source change.
// Error convention kept from the reference (RTERROR/LAUNCHERROR,
// cuda/GpuData.h:40-72): print, reset the device, exit(-1).
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/adgpu_b200.h"

struct GpuData;   // the reference's struct; byte-identical to adgpu_gpudata

static void die_on(adgpu_status st, const char* what)
{
	if (st == ADGPU_OK) return;
	printf("Error: %s launching kernel %s\n", adgpu_last_error(), what);
	cudaDeviceReset();
	exit(-1);
}

void SetKernelsGpuData(GpuData* pData)
{
	die_on(adgpu_set_kernels_gpu_data(reinterpret_cast<const adgpu_gpudata*>(pData)), "SetKernelsGpuData");
}

void GetKernelsGpuData(GpuData* pData)
{
	die_on(adgpu_get_kernels_gpu_data(reinterpret_cast<adgpu_gpudata*>(pData)), "GetKernelsGpuData");
}

void gpu_calc_initpop(uint32_t blocks, uint32_t threadsPerBlock, float* pConformations_current, float* pEnergies_current)
{
	die_on(adgpu_calc_initpop(blocks, threadsPerBlock, pConformations_current, pEnergies_current), "gpu_calc_initpop_kernel");
}

void gpu_sum_evals(uint32_t blocks, uint32_t threadsPerBlock)
{
	die_on(adgpu_sum_evals(blocks, threadsPerBlock), "gpu_sum_evals_kernel");
}

void gpu_gen_and_eval_newpops(uint32_t blocks, uint32_t threadsPerBlock, float* pMem_conformations_current,
                              float* pMem_energies_current, float* pMem_conformations_next, float* pMem_energies_next)
{
	die_on(adgpu_gen_and_eval_newpops(blocks, threadsPerBlock, pMem_conformations_current, pMem_energies_current,
	                                  pMem_conformations_next, pMem_energies_next),
	       "gpu_gen_and_eval_newpops_kernel");
}

void gpu_perform_LS(uint32_t blocks, uint32_t threads, float* pMem_conformations_next, float* pMem_energies_next)
{
	die_on(adgpu_perform_ls(blocks, threads, pMem_conformations_next, pMem_energies_next), "gpu_perform_LS_kernel");
}

void gpu_gradient_minAD(uint32_t blocks, uint32_t threads, float* pMem_conformations_next, float* pMem_energies_next)
{
	die_on(adgpu_gradient_minad(blocks, threads, pMem_conformations_next, pMem_energies_next), "gpu_gradient_minAD_kernel");
}

void gpu_gradient_minAdam(uint32_t blocks, uint32_t threads, float* pMem_conformations_next, float* pMem_energies_next)
{
	die_on(adgpu_gradient_minadam(blocks, threads, pMem_conformations_next, pMem_energies_next), "gpu_gradient_minAdam_kernel");
}
