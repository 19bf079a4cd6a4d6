/*
 * adgpu_oracle.h -- CPU restatement of AutoDock-GPU's LGA hot path.
 *
 * TEST INFRASTRUCTURE: the checker the CUDA engine is compared against
 * (tests/, __graft_entry__.smoke(), and bench.py's CPU-baseline leg only).
 * The product never links it.  Parity of this restatement with the
 * reference's own kernel source is pinned by tests/test_oracle_pins.py, which
 * runs both on the same inputs (oracle/_ref builds the reference's sources
 * for the CPU) and by the committed vectors in tests/golden/.
 *
 * Tables are the reference's (see include/adgpu_b200.h); all pointers inside
 * the adgpu_gpudata passed here are HOST pointers.  Launch semantics follow
 * the reference: `blocks` blocks, and `threads` is the reference block size
 * that fixes which per-thread LCG state each draw consumes
 * (prng_states[block*threads + lane], cuda/auxiliary_genetic.cu:37).
 */
#ifndef ADGPU_ORACLE_H
#define ADGPU_ORACLE_H

#include "adgpu_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Energy (gradient == NULL) or energy + gene gradient of one genotype:
 * gpu_calc_energy (cuda/calcenergy.cu:114-453) and gpu_calc_energrad
 * (cuda/calcMergeEneGra.cu:48-900).  terms (nullable) receives
 * [E_inter_type, E_inter_elec, E_inter_desolv, E_intra_vdw_hb, E_intra_elec,
 *  E_intra_desolv, E_intra_cg_g0, n_out_of_grid]. */
void oracle_score(const adgpu_gpudata* d, const float* genotype, float* energy, float* gradient, float* terms);

/* Batch of n genotypes (stride 64) over `nthreads` OS threads. */
void oracle_score_batch(const adgpu_gpudata* d, uint32_t n, const float* genotypes, float* energies,
                        float* gradients, int nthreads);

void oracle_calc_initpop(const adgpu_gpudata* d, uint32_t blocks, float* conf_cur, float* e_cur, int nthreads);
void oracle_sum_evals(const adgpu_gpudata* d, uint32_t blocks);
void oracle_gen_and_eval_newpops(const adgpu_gpudata* d, uint32_t blocks, uint32_t threads,
                                 const float* conf_cur, const float* e_cur, float* conf_next, float* e_next,
                                 int nthreads);
void oracle_perform_ls(const adgpu_gpudata* d, uint32_t blocks, uint32_t threads,
                       float* conf_next, float* e_next, int nthreads);
void oracle_gradient_minad(const adgpu_gpudata* d, uint32_t blocks, uint32_t threads,
                           float* conf_next, float* e_next, int nthreads);
void oracle_gradient_minadam(const adgpu_gpudata* d, uint32_t blocks, uint32_t threads,
                             float* conf_next, float* e_next, int nthreads);
void oracle_gradient_minfire(const adgpu_gpudata* d, uint32_t blocks, uint32_t threads,
                             float* conf_next, float* e_next, int nthreads);

#ifdef __cplusplus
}
#endif

#endif
