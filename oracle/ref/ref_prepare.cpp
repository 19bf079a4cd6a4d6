/*
 * ref_prepare.cpp -- drives the reference's own host front end (compiled from
 * host/src/*.cpp of AutoDock-GPU where they lie) to turn .fld/.map/.pdbqt
 * inputs plus a command line into the exact tables the reference hands to
 * its kernel API.  TEST INFRASTRUCTURE ONLY (oracle side).
 *
 * Sequence restated from the reference:
 *   initial_commandpars + get_filelist        host/src/main.cpp:104-107
 *   setup()                                   host/src/main.cpp:333 -> host/src/setup.cpp:60
 *   gen_initpop_and_reflig, LocalRNG seeds    host/src/performdocking.cpp.Cuda:302-317
 *   prepare_const_fields_for_gpu              host/src/performdocking.cpp.Cuda:352-361
 *   GpuDockparameters fill                    host/src/performdocking.cpp.Cuda:413-463
 */
#include <cstring>
#include <string>
#include <vector>
#include <cstdint>
#include "filelist.hpp"
#include "processgrid.h"
#include "processligand.h"
#include "getparameters.h"
#include "setup.hpp"
#include "calcenergy.h"

/* GpuDockparameters, cuda/GpuData.h:74-110 (kept byte-identical). */
typedef struct {
	int num_of_atoms, true_ligand_atoms, num_of_atypes, num_of_map_atypes, num_of_intraE_contributors;
	int gridsize_x, gridsize_y, gridsize_z, gridsize_x_times_y, gridsize_x_times_y_times_z;
	float grid_spacing;
	int rotbondlist_length;
	float coeff_elec, elec_min_distance, coeff_desolv;
	int pop_size, num_of_genes;
	float tournament_rate, crossover_rate, mutation_rate, abs_max_dmov, abs_max_dang, lsearch_rate, smooth;
	unsigned int num_of_lsentities;
	float rho_lower_bound, base_dmov_mul_sqrt3, base_dang_mul_sqrt3;
	unsigned int cons_limit, max_num_of_iters;
	float qasp, adam_beta1, adam_beta2, adam_epsilon;
} RefDockpars;

struct RefJob {
	RefDockpars dockpars;
	kernelconstant_interintra interintra;
	kernelconstant_intracontrib intracontrib;
	kernelconstant_intra intra;
	kernelconstant_rotlist rotlist;
	kernelconstant_conform conform;
	kernelconstant_grads grads;
	std::vector<float> grid;
	std::vector<float> initpop;
	std::vector<uint32_t> prng;
	int num_runs = 0;
	int num_rotbonds = 0;
	int num_rotcyc = 0;
	unsigned long nev = 0;
	unsigned long ngen = 0;
	char lsmet[8] = {0};
	float grid_origin[3] = {0, 0, 0};
	float grid_size_angstrom[3] = {0, 0, 0};
	std::vector<int32_t> bonds;        // [N*N] bond matrix of the prepared ligand
	std::vector<int32_t> rigid;        // [N] rigid structure ids
	std::vector<int32_t> contrib;      // [N*N] intramolecular contributor matrix
};

/* GpuData layout of cuda/GpuData.h:112-136, with plain pointer members. */
struct RefGpuData {
	int devnum, devid, preallocated_gridsize;
	RefDockpars dockpars;
	void* pKerconst_interintra;
	void* pKerconst_intracontrib;
	void* pKerconst_intra;
	void* pKerconst_rotlist;
	void* pKerconst_conform;
	void* pKerconst_grads;
	float* pMem_fgrids;
	int* pMem_evals_of_new_entities;
	int* pMem_gpu_evals_of_runs;
	uint32_t* pMem_prng_states;
	int* pMem_rotbonds_const;
	int* pMem_rotbonds_atoms_const;
	int* pMem_num_rotating_atoms_per_rotbond_const;
	unsigned int warpmask, warpbits;
};

extern "C" void adgpu_ref_set_gpudata(const void* data);

extern "C" {

typedef struct {
	int num_of_atoms, true_ligand_atoms, num_of_rotbonds, num_of_genes, num_of_intraE_contributors;
	int num_of_rotcyc, pop_size, num_of_runs, num_of_lsentities, num_of_map_atypes;
	int gridsize[3];
	float spacing;
	float grid_origin[3];
	unsigned long nev, ngen;
	char lsmet[8];
} adgpu_ref_info;

void* adgpu_ref_job_create(int argc, char** argv)
{
	FileList filelist;
	Dockpars initial_pars;
	Gridinfo initial_grid;
	if (initial_commandpars(&argc, argv, &initial_pars, &initial_grid, filelist) != 0) return nullptr;
	if (get_filelist(&argc, argv, &initial_pars, &initial_grid, filelist) != 0) return nullptr;
	Dockpars mypars = initial_pars;
	Gridinfo* mygrid = &initial_grid;
	if (filelist.used) {
		mypars = filelist.mypars[0];
		mygrid = &filelist.mygrids[mypars.filelist_grid_idx];
	}
	Liganddata* lig_init = new Liganddata;
	Liganddata* xray = new Liganddata;
	if (setup(mygrid, &mypars, *lig_init, *xray, filelist, 0, argc, argv) != 0) {
		delete lig_init; delete xray; return nullptr;
	}
	RefJob* job = new RefJob;
	job->num_runs = (int)mypars.num_of_runs;
	size_t npop = (size_t)mypars.num_of_runs * mypars.pop_size;
	job->initpop.assign(npop * GENOTYPE_LENGTH_IN_GLOBMEM, 0.0f);
	Liganddata* lig = new Liganddata;
	*lig = *lig_init;
	gen_initpop_and_reflig(&mypars, job->initpop.data(), lig, mygrid);
	job->prng.resize(npop * NUM_OF_THREADS_PER_BLOCK);
	LocalRNG r(mypars.seed);
	for (size_t i = 0; i < job->prng.size(); i++) job->prng[i] = r.random_uint();
	if (prepare_const_fields_for_gpu(lig, &mypars, &job->interintra, &job->intracontrib, &job->intra,
	                                 &job->rotlist, &job->conform, &job->grads) != 0) {
		delete lig; delete lig_init; delete xray; delete job; return nullptr;
	}
	job->grid.assign(mygrid->grids.begin(), mygrid->grids.end());
	RefDockpars& d = job->dockpars;
	memset(&d, 0, sizeof(d));
	d.num_of_atoms = lig->num_of_atoms;
	d.true_ligand_atoms = (int)lig->true_ligand_atoms;
	d.num_of_atypes = lig->num_of_atypes;
	d.num_of_map_atypes = mygrid->num_of_map_atypes;
	d.num_of_intraE_contributors = (int)lig->num_of_intraE_contributors;
	d.gridsize_x = mygrid->size_xyz[0];
	d.gridsize_y = mygrid->size_xyz[1];
	d.gridsize_z = mygrid->size_xyz[2];
	d.gridsize_x_times_y = d.gridsize_x * d.gridsize_y;
	d.gridsize_x_times_y_times_z = d.gridsize_x * d.gridsize_y * d.gridsize_z;
	d.grid_spacing = (float)mygrid->spacing;
	d.rotbondlist_length = (int)NUM_OF_THREADS_PER_BLOCK * lig->num_of_rotcyc;
	d.coeff_elec = (float)mypars.coeffs.scaled_AD4_coeff_elec;
	d.elec_min_distance = (float)mypars.elec_min_distance;
	d.coeff_desolv = (float)mypars.coeffs.AD4_coeff_desolv;
	d.pop_size = (int)mypars.pop_size;
	d.num_of_genes = lig->num_of_rotbonds + 6;
	d.tournament_rate = mypars.tournament_rate / 100.0f;
	d.crossover_rate = mypars.crossover_rate / 100.0f;
	d.mutation_rate = mypars.mutation_rate / 100.f;
	d.abs_max_dang = mypars.abs_max_dang;
	d.abs_max_dmov = mypars.abs_max_dmov;
	d.qasp = mypars.qasp;
	d.smooth = mypars.smooth;
	d.lsearch_rate = mypars.lsearch_rate;
	d.adam_beta1 = mypars.adam_beta1;
	d.adam_beta2 = mypars.adam_beta2;
	d.adam_epsilon = mypars.adam_epsilon;
	if (d.lsearch_rate != 0.0f) {
		d.num_of_lsentities = (unsigned int)(mypars.lsearch_rate / 100.0 * mypars.pop_size + 0.5);
		d.rho_lower_bound = mypars.rho_lower_bound;
		d.base_dmov_mul_sqrt3 = mypars.base_dmov_mul_sqrt3;
		d.base_dang_mul_sqrt3 = mypars.base_dang_mul_sqrt3;
		d.cons_limit = (unsigned int)mypars.cons_limit;
		d.max_num_of_iters = (unsigned int)mypars.max_num_of_iters;
	}
	job->num_rotbonds = lig->num_of_rotbonds;
	job->num_rotcyc = lig->num_of_rotcyc;
	job->nev = mypars.num_of_energy_evals;
	job->ngen = mypars.num_of_generations;
	strncpy(job->lsmet, mypars.ls_method, sizeof(job->lsmet) - 1);
	for (int i = 0; i < 3; i++) job->grid_origin[i] = (float)mygrid->origo_real_xyz[i];
	{
		int n = lig->num_of_atoms;
		job->bonds.resize((size_t)n * n); job->contrib.resize((size_t)n * n); job->rigid.resize(n);
		for (int a = 0; a < n; a++) {
			job->rigid[a] = lig->atom_rigid_structures[a];
			for (int b = 0; b < n; b++) {
				job->bonds[(size_t)a * n + b] = lig->bonds[a][b];
				job->contrib[(size_t)a * n + b] = lig->intraE_contributors[a][b];
			}
		}
	}
	delete lig; delete lig_init; delete xray;
	return job;
}

void adgpu_ref_job_free(void* h) { delete (RefJob*)h; }

int adgpu_ref_job_info(void* h, adgpu_ref_info* out)
{
	RefJob* j = (RefJob*)h;
	memset(out, 0, sizeof(*out));
	out->num_of_atoms = j->dockpars.num_of_atoms;
	out->true_ligand_atoms = j->dockpars.true_ligand_atoms;
	out->num_of_rotbonds = j->num_rotbonds;
	out->num_of_genes = j->dockpars.num_of_genes;
	out->num_of_intraE_contributors = j->dockpars.num_of_intraE_contributors;
	out->num_of_rotcyc = j->num_rotcyc;
	out->pop_size = j->dockpars.pop_size;
	out->num_of_runs = j->num_runs;
	out->num_of_lsentities = (int)j->dockpars.num_of_lsentities;
	out->num_of_map_atypes = j->dockpars.num_of_map_atypes;
	out->gridsize[0] = j->dockpars.gridsize_x;
	out->gridsize[1] = j->dockpars.gridsize_y;
	out->gridsize[2] = j->dockpars.gridsize_z;
	out->spacing = j->dockpars.grid_spacing;
	for (int i = 0; i < 3; i++) out->grid_origin[i] = j->grid_origin[i];
	out->nev = j->nev;
	out->ngen = j->ngen;
	memcpy(out->lsmet, j->lsmet, sizeof(out->lsmet));
	return 0;
}

/* Pointer to, and size of, one of the job's tables. */
void* adgpu_ref_job_blob(void* h, const char* name, size_t* nbytes)
{
	RefJob* j = (RefJob*)h;
	std::string n(name);
#define BLOB(key, ptr, sz) if (n == key) { *nbytes = (sz); return (void*)(ptr); }
	BLOB("dockpars", &j->dockpars, sizeof(j->dockpars));
	BLOB("interintra", &j->interintra, sizeof(j->interintra));
	BLOB("intracontrib", &j->intracontrib, sizeof(j->intracontrib));
	BLOB("intra", &j->intra, sizeof(j->intra));
	BLOB("rotlist", &j->rotlist, sizeof(j->rotlist));
	BLOB("conform", &j->conform, sizeof(j->conform));
	BLOB("grads", &j->grads, sizeof(j->grads));
	BLOB("grid", j->grid.data(), j->grid.size() * sizeof(float));
	BLOB("initpop", j->initpop.data(), j->initpop.size() * sizeof(float));
	BLOB("prng", j->prng.data(), j->prng.size() * sizeof(uint32_t));
	BLOB("bonds", j->bonds.data(), j->bonds.size() * sizeof(int32_t));
	BLOB("rigid", j->rigid.data(), j->rigid.size() * sizeof(int32_t));
	BLOB("contrib", j->contrib.data(), j->contrib.size() * sizeof(int32_t));
#undef BLOB
	*nbytes = 0;
	return nullptr;
}

/* Points the emulated kernels at this job's tables (host memory stands in
 * for device memory), with caller-owned PRNG states and eval counters, and
 * an optional override of the docking parameters. */
int adgpu_ref_job_bind(void* h, const void* dockpars_override, uint32_t* prng_states,
                       int* evals_of_new_entities, int* evals_of_runs)
{
	RefJob* j = (RefJob*)h;
	RefGpuData g;
	memset(&g, 0, sizeof(g));
	g.dockpars = dockpars_override ? *(const RefDockpars*)dockpars_override : j->dockpars;
	g.pKerconst_interintra = &j->interintra;
	g.pKerconst_intracontrib = &j->intracontrib;
	g.pKerconst_intra = &j->intra;
	g.pKerconst_rotlist = &j->rotlist;
	g.pKerconst_conform = &j->conform;
	g.pKerconst_grads = &j->grads;
	g.pMem_fgrids = j->grid.data();
	g.pMem_evals_of_new_entities = evals_of_new_entities;
	g.pMem_gpu_evals_of_runs = evals_of_runs;
	g.pMem_prng_states = prng_states;
	g.pMem_rotbonds_const = j->grads.rotbonds;
	g.pMem_rotbonds_atoms_const = j->grads.rotbonds_atoms;
	g.pMem_num_rotating_atoms_per_rotbond_const = j->grads.num_rotating_atoms_per_rotbond;
	g.warpmask = 31;
	g.warpbits = 5;
	adgpu_ref_set_gpudata(&g);
	return 0;
}

size_t adgpu_ref_sizeof_refgpudata(void) { return sizeof(RefGpuData); }

}  // extern "C"
