// ref_cuda_tu.cu -- the reference's CUDA kernel API (cuda/kernels.cu and the
// kernel files it includes), compiled unchanged with nvcc for sm_100a, with C
// entry points for the test suite and the measurement scripts: this is the
// reference's own GPU path on the same B200, used to compare results and to
// time the kernels the engine replaces.  TEST INFRASTRUCTURE ONLY.
#include "kernels.cu"

__global__ void adgpu_refcuda_score_kernel(const float* genotypes, float* energies, float* gradients)
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
void adgpu_refcuda_set_gpudata(void* d) { SetKernelsGpuData((GpuData*)d); }
int adgpu_refcuda_score(uint32_t n, const float* g, float* e, float* gr)
{
	adgpu_refcuda_score_kernel<<<n, NUM_OF_THREADS_PER_BLOCK>>>(g, e, gr);
	return (int)cudaDeviceSynchronize();
}
void adgpu_refcuda_calc_initpop(uint32_t b, uint32_t t, float* c, float* e) { gpu_calc_initpop(b, t, c, e); }
void adgpu_refcuda_sum_evals(uint32_t b, uint32_t t) { gpu_sum_evals(b, t); }
void adgpu_refcuda_gen_and_eval_newpops(uint32_t b, uint32_t t, float* cc, float* ec, float* cn, float* en)
{
	gpu_gen_and_eval_newpops(b, t, cc, ec, cn, en);
}
void adgpu_refcuda_perform_ls(uint32_t b, uint32_t t, float* c, float* e) { gpu_perform_LS(b, t, c, e); }
void adgpu_refcuda_gradient_minad(uint32_t b, uint32_t t, float* c, float* e) { gpu_gradient_minAD(b, t, c, e); }
void adgpu_refcuda_gradient_minadam(uint32_t b, uint32_t t, float* c, float* e) { gpu_gradient_minAdam(b, t, c, e); }
}
