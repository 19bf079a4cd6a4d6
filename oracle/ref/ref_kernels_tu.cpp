/*
 * ref_kernels_tu.cpp -- builds the reference's own CUDA kernel sources
 * (cuda/kernels.cu and everything it includes, cuda/kernels.cu:142-151) as
 * host C++ under the SIMT emulator (simt_shim.h), and exports them with C
 * linkage for the test suite.  TEST INFRASTRUCTURE ONLY.
 *
 * The recipe in oracle/Makefile preprocesses this file, rewrites every
 * `kernel<<<blocks, threads>>>(args);` launch of the reference into
 * `adgpu_ref_launch(blocks, threads, [&]{ kernel(args); });` and compiles the
 * result; the reference sources are read where they lie and no copy of them
 * is written anywhere.
 */
#include "simt_shim.h"
#include "kernels.cu"

/* Batch scorer around the reference's device functions: block b scores
 * genotype b with gpu_calc_energy (cuda/calcenergy.cu:114) or
 * gpu_calc_energrad (cuda/calcMergeEneGra.cu:48). */
__global__ void adgpu_ref_score_kernel(const float* genotypes, float* energies, float* gradients)
{
	__shared__ float3 calc_coords[MAX_NUM_OF_ATOMS];
	__shared__ int3 cart_grad[MAX_NUM_OF_ATOMS];
	__shared__ float genotype[ACTUAL_GENOTYPE_LENGTH];
	__shared__ float grad[ACTUAL_GENOTYPE_LENGTH];
	__shared__ float acc;
	float energy = 0.0f;
	int run_id = 0;
	for (int i = threadIdx.x; i < cData.dockpars.num_of_genes; i += blockDim.x)
		genotype[i] = genotypes[blockIdx.x * GENOTYPE_LENGTH_IN_GLOBMEM + i];
	__syncthreads();
	if (gradients == nullptr) {
		gpu_calc_energy(genotype, energy, run_id, calc_coords, &acc);
	} else {
		gpu_calc_energrad(genotype, energy, run_id, calc_coords, cart_grad, grad, &acc);
		for (int i = threadIdx.x; i < cData.dockpars.num_of_genes; i += blockDim.x)
			gradients[blockIdx.x * GENOTYPE_LENGTH_IN_GLOBMEM + i] = grad[i];
	}
	if (threadIdx.x == 0) energies[blockIdx.x] = energy;
}

extern "C" {

void adgpu_ref_set_gpudata(const void* data) { SetKernelsGpuData((GpuData*)data); }
void adgpu_ref_get_gpudata(void* data) { memcpy(data, &cpuData, sizeof(GpuData)); }
size_t adgpu_ref_sizeof_gpudata(void) { return sizeof(GpuData); }

void adgpu_ref_score(uint32_t n, uint32_t threads, const float* genotypes, float* energies, float* gradients)
{
	adgpu_ref_launch(n, threads, [&] { adgpu_ref_score_kernel(genotypes, energies, gradients); });
}

void adgpu_ref_calc_initpop(uint32_t blocks, uint32_t threads, float* conf, float* e)
{
	gpu_calc_initpop(blocks, threads, conf, e);
}

void adgpu_ref_sum_evals(uint32_t blocks, uint32_t threads) { gpu_sum_evals(blocks, threads); }

void adgpu_ref_gen_and_eval_newpops(uint32_t blocks, uint32_t threads, float* cc, float* ec, float* cn, float* en)
{
	gpu_gen_and_eval_newpops(blocks, threads, cc, ec, cn, en);
}

void adgpu_ref_perform_ls(uint32_t blocks, uint32_t threads, float* cn, float* en) { gpu_perform_LS(blocks, threads, cn, en); }
void adgpu_ref_gradient_minad(uint32_t blocks, uint32_t threads, float* cn, float* en) { gpu_gradient_minAD(blocks, threads, cn, en); }
void adgpu_ref_gradient_minadam(uint32_t blocks, uint32_t threads, float* cn, float* en) { gpu_gradient_minAdam(blocks, threads, cn, en); }

}
