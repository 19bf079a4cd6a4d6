/*
 * ref_fire_tu.cpp -- builds the reference's OpenCL FIRE local search
 * (device/kernel_fire.cl, gradient_minFire) with the device functions the
 * reference's OpenCL program puts before it (the order of
 * stringify_ocl_krnls.sh: defines.h, calcenergy_basic.h, auxiliary_genetic.cl,
 * calcenergy.cl, calcgradient.cl, calcMergedEneGra.cl) as host C++ under the
 * SIMT emulator (ocl_shim.h), and exports it with C linkage for the test
 * suite.  TEST INFRASTRUCTURE ONLY.
 *
 * The recipe in oracle/Makefile preprocesses this file, rewrites the
 * work-group declarations `__local T name[...];` of the kernel into
 * `static thread_local` ones and `(float4)(` vector literals into
 * make_float4( calls, drops the remaining `__local` qualifiers, and compiles
 * the result; the reference sources are read where they lie.
 */
#include "ocl_shim.h"
#include "adgpu_b200.h"          /* adgpu_gpudata: GpuData's layout (cuda/GpuData.h:112-136) */
#include "calcenergy_basic.h"
#include "auxiliary_genetic.cl"
#include "calcenergy.cl"
#include "calcgradient.cl"
#include "calcMergedEneGra.cl"

/* FIRE's first gradient (kernel_fire.cl:318-358) comes from calcgradient.cl's
 * gpu_calc_gradient, which, unlike the energy scorers, never loads the
 * reference coordinates into calc_coords (calcgradient.cl:160-258 rotates
 * whatever the kernel's __local calc_coords holds, and kernel_fire.cl writes
 * nothing there first): on a device that is what an earlier work-group left
 * in local memory, here what the previous block on this host thread left.
 * The overload below (selected because the kernel passes its int gradient
 * arrays, which OpenCL C converts to the float accumulators implicitly)
 * either keeps that call (adgpu_ref_fire_first_gradient = 0) or takes the
 * first gradient from the reference's merged scorer gpu_calc_energrad on the
 * same genotype (= 1, the default), which is what the engine's FIRE does. */
extern "C" int adgpu_ref_fire_first_gradient;
int adgpu_ref_fire_first_gradient = 1;

static inline void gpu_calc_gradient(int rl, int na, int tla, int gx, int gy, int gz, uint gxy, uint gxyz,
                                     const float* fg, int nat, int nmat, int nie, float sp, float ce, float emd,
                                     float qasp, float cd, float sm, float* geno, float* energy, int* run_id,
                                     float4* coords, kernelconstant_interintra* ii, const kernelconstant_intracontrib* ic,
                                     kernelconstant_intra* in, kernelconstant_rotlist* rl_, kernelconstant_conform* cf,
                                     int* rb, const int* rba, int* nrr, int ng, int* ix, int* iy, int* iz,
                                     float* fx, float* fy, float* fz, float* grad)
{
	__local float partial_energies[NUM_OF_THREADS_PER_BLOCK];
	__local float first_energy;
	if (adgpu_ref_fire_first_gradient)
		gpu_calc_energrad(rl, na, tla, gx, gy, gz, gxy, gxyz, fg, nat, nmat, nie, sp, ce, emd, qasp, cd, sm, geno,
		                  &first_energy, run_id, coords, partial_energies, ii, ic, in, rl_, cf, rb, rba, nrr, ng,
		                  ix, iy, iz, fx, fy, fz, grad);
	else
		gpu_calc_gradient(rl, na, tla, gx, gy, gz, gxy, gxyz, fg, nat, nmat, nie, sp, ce, emd, qasp, cd, sm, geno,
		                  energy, run_id, coords, ii, ic, in, rl_, cf, rb, rba, nrr, ng, (float*)ix, (float*)iy,
		                  (float*)iz, fx, fy, fz, grad);
}

#include "kernel_fire.cl"

extern "C" void adgpu_ref_fire(const void* gpudata, uint32_t blocks, uint32_t threads, float* conf, float* energies)
{
	const adgpu_gpudata& d = *static_cast<const adgpu_gpudata*>(gpudata);
	const adgpu_dockpars& p = d.dockpars;
	adgpu_ref_launch(blocks, threads, [&] {
		gradient_minFire(p.num_of_atoms, p.true_ligand_atoms, p.num_of_atypes, p.num_of_map_atypes,
		                 p.num_of_intraE_contributors, p.gridsize_x, p.gridsize_y, p.gridsize_z,
		                 p.gridsize_x_times_y, p.gridsize_x_times_y_times_z, p.grid_spacing, d.pMem_fgrids,
		                 p.rotbondlist_length, p.coeff_elec, p.elec_min_distance, p.coeff_desolv,
		                 conf, energies, d.pMem_evals_of_new_entities, d.pMem_prng_states,
		                 p.pop_size, p.num_of_genes, p.lsearch_rate, p.num_of_lsentities, p.max_num_of_iters,
		                 p.qasp, p.smooth,
		                 (kernelconstant_interintra*)d.pKerconst_interintra,
		                 (const kernelconstant_intracontrib*)d.pKerconst_intracontrib,
		                 (kernelconstant_intra*)d.pKerconst_intra,
		                 (kernelconstant_rotlist*)d.pKerconst_rotlist,
		                 (kernelconstant_conform*)d.pKerconst_conform,
		                 d.pMem_rotbonds_const, d.pMem_rotbonds_atoms_const,
		                 d.pMem_num_rotating_atoms_per_rotbond_const);
	});
}

/* The reference's OpenCL merged scorer (calcMergedEneGra.cl, gpu_calc_energrad)
 * on n genotypes, block b scoring genotype b: energies and gene gradients. */
static void adgpu_ref_ocl_score_block(const adgpu_gpudata& d, const float* genotypes, float* energies, float* grads)
{
	const adgpu_dockpars& p = d.dockpars;
	__local float genotype[ACTUAL_GENOTYPE_LENGTH];
	__local float energy;
	__local int run_id;
	__local float4 calc_coords[MAX_NUM_OF_ATOMS];
	__local float partial_energies[NUM_OF_THREADS_PER_BLOCK];
	__local int gx[MAX_NUM_OF_ATOMS];
	__local int gy[MAX_NUM_OF_ATOMS];
	__local int gz[MAX_NUM_OF_ATOMS];
	__local float fx[MAX_NUM_OF_ATOMS];
	__local float fy[MAX_NUM_OF_ATOMS];
	__local float fz[MAX_NUM_OF_ATOMS];
	__local float gradient[ACTUAL_GENOTYPE_LENGTH];
	const unsigned b = get_group_id(0), t = get_local_id(0);
	for (int i = t; i < p.num_of_genes; i += NUM_OF_THREADS_PER_BLOCK) genotype[i] = genotypes[b * GENOTYPE_LENGTH_IN_GLOBMEM + i];
	if (t == 0) run_id = 0;
	barrier(CLK_LOCAL_MEM_FENCE);
	gpu_calc_energrad(p.rotbondlist_length, p.num_of_atoms, p.true_ligand_atoms, p.gridsize_x, p.gridsize_y,
	                  p.gridsize_z, p.gridsize_x_times_y, p.gridsize_x_times_y_times_z, d.pMem_fgrids, p.num_of_atypes,
	                  p.num_of_map_atypes, p.num_of_intraE_contributors, p.grid_spacing, p.coeff_elec,
	                  p.elec_min_distance, p.qasp, p.coeff_desolv, p.smooth, genotype, &energy, &run_id, calc_coords,
	                  partial_energies, (kernelconstant_interintra*)d.pKerconst_interintra,
	                  (const kernelconstant_intracontrib*)d.pKerconst_intracontrib,
	                  (kernelconstant_intra*)d.pKerconst_intra, (kernelconstant_rotlist*)d.pKerconst_rotlist,
	                  (kernelconstant_conform*)d.pKerconst_conform, d.pMem_rotbonds_const, d.pMem_rotbonds_atoms_const,
	                  d.pMem_num_rotating_atoms_per_rotbond_const, p.num_of_genes, gx, gy, gz, fx, fy, fz, gradient);
	barrier(CLK_LOCAL_MEM_FENCE);
	for (int i = t; i < p.num_of_genes; i += NUM_OF_THREADS_PER_BLOCK) grads[b * GENOTYPE_LENGTH_IN_GLOBMEM + i] = gradient[i];
	if (t == 0) energies[b] = energy;
}

extern "C" void adgpu_ref_ocl_score(const void* gpudata, uint32_t n, const float* genotypes, float* energies, float* grads)
{
	const adgpu_gpudata& d = *static_cast<const adgpu_gpudata*>(gpudata);
	adgpu_ref_launch(n, NUM_OF_THREADS_PER_BLOCK, [&] { adgpu_ref_ocl_score_block(d, genotypes, energies, grads); });
}
